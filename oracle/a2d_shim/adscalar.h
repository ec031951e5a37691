// Forward-mode scalar with N directional derivatives, restating the interface of
// A2D's ADScalar (github.com/smdogroup/a2d; the reference pins no version, only
// an include path, Makefile.in:2-3) as element/FEKernels.h and
// element/LagrangeShapeFuncs.h use it: public `value` and `deriv[N]`, construction
// and assignment from a plain value (derivatives cleared), and the arithmetic
// operators with the usual first-order rules.
//
// TEST INFRASTRUCTURE ONLY: it lets the reference's own CPU assembly compile as
// oracle/_ref (oracle/Makefile, target `ref`) so that the oracle restatement can
// be compared with it.  Nothing in the library under gpu-fem-project_b200/ uses it.
#pragma once

#include <cmath>

namespace A2D {

template <class T, int N>
class ADScalar {
 public:
  T value;
  T deriv[N];

  ADScalar(const T v = T(0)) : value(v) {
    for (int i = 0; i < N; i++) deriv[i] = T(0);
  }
  ADScalar &operator=(const T &v) {
    value = v;
    for (int i = 0; i < N; i++) deriv[i] = T(0);
    return *this;
  }
  ADScalar &operator+=(const ADScalar &b) {
    value += b.value;
    for (int i = 0; i < N; i++) deriv[i] += b.deriv[i];
    return *this;
  }
  ADScalar &operator-=(const ADScalar &b) {
    value -= b.value;
    for (int i = 0; i < N; i++) deriv[i] -= b.deriv[i];
    return *this;
  }
  ADScalar &operator*=(const ADScalar &b) {
    for (int i = 0; i < N; i++) deriv[i] = deriv[i] * b.value + value * b.deriv[i];
    value *= b.value;
    return *this;
  }
};

template <class T, int N>
ADScalar<T, N> operator-(const ADScalar<T, N> &a) {
  ADScalar<T, N> r(-a.value);
  for (int i = 0; i < N; i++) r.deriv[i] = -a.deriv[i];
  return r;
}
template <class T, int N>
ADScalar<T, N> operator+(const ADScalar<T, N> &a, const ADScalar<T, N> &b) {
  ADScalar<T, N> r(a.value + b.value);
  for (int i = 0; i < N; i++) r.deriv[i] = a.deriv[i] + b.deriv[i];
  return r;
}
template <class T, int N>
ADScalar<T, N> operator-(const ADScalar<T, N> &a, const ADScalar<T, N> &b) {
  ADScalar<T, N> r(a.value - b.value);
  for (int i = 0; i < N; i++) r.deriv[i] = a.deriv[i] - b.deriv[i];
  return r;
}
template <class T, int N>
ADScalar<T, N> operator*(const ADScalar<T, N> &a, const ADScalar<T, N> &b) {
  ADScalar<T, N> r(a.value * b.value);
  for (int i = 0; i < N; i++) r.deriv[i] = a.deriv[i] * b.value + a.value * b.deriv[i];
  return r;
}
template <class T, int N>
ADScalar<T, N> operator/(const ADScalar<T, N> &a, const ADScalar<T, N> &b) {
  const T inv = T(1) / b.value;
  ADScalar<T, N> r(a.value * inv);
  for (int i = 0; i < N; i++) r.deriv[i] = (a.deriv[i] - r.value * b.deriv[i]) * inv;
  return r;
}
// mixed with a plain value
template <class T, int N>
ADScalar<T, N> operator+(const ADScalar<T, N> &a, const T &b) {
  ADScalar<T, N> r = a;
  r.value += b;
  return r;
}
template <class T, int N>
ADScalar<T, N> operator+(const T &a, const ADScalar<T, N> &b) {
  return b + a;
}
template <class T, int N>
ADScalar<T, N> operator-(const ADScalar<T, N> &a, const T &b) {
  ADScalar<T, N> r = a;
  r.value -= b;
  return r;
}
template <class T, int N>
ADScalar<T, N> operator-(const T &a, const ADScalar<T, N> &b) {
  return -(b - a);
}
template <class T, int N>
ADScalar<T, N> operator*(const ADScalar<T, N> &a, const T &b) {
  ADScalar<T, N> r(a.value * b);
  for (int i = 0; i < N; i++) r.deriv[i] = a.deriv[i] * b;
  return r;
}
template <class T, int N>
ADScalar<T, N> operator*(const T &a, const ADScalar<T, N> &b) {
  ADScalar<T, N> r(a * b.value);
  for (int i = 0; i < N; i++) r.deriv[i] = a * b.deriv[i];
  return r;
}
template <class T, int N>
ADScalar<T, N> operator/(const ADScalar<T, N> &a, const T &b) {
  ADScalar<T, N> r(a.value / b);
  for (int i = 0; i < N; i++) r.deriv[i] = a.deriv[i] / b;
  return r;
}
// fused multiply-add in the value, first-order rule in the derivatives (the
// generic lagrangePoly1d template evaluates its polynomial with fma)
template <class T, int N>
ADScalar<T, N> fma(const ADScalar<T, N> &a, const ADScalar<T, N> &b, const ADScalar<T, N> &c) {
  ADScalar<T, N> r(std::fma(a.value, b.value, c.value));
  for (int i = 0; i < N; i++) r.deriv[i] = a.deriv[i] * b.value + a.value * b.deriv[i] + c.deriv[i];
  return r;
}

}  // namespace A2D
