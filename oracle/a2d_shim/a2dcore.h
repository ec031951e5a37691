// The subset of A2D's dense-matrix and reverse-mode AD interface that
// element/FEKernels.h uses, restated from its documented semantics (A2D,
// github.com/smdogroup/a2d; the reference pins no version, only an include
// path, Makefile.in:2-3).  Call sites: Mat / zero / get_data / operator() and []
// (FEKernels.h:20-42, 230-284, 317-508), MatMatMult<MatOp, MatOp>
// (:122-123, 283, 463), MatInv / MatDet for 2x2 (:356-359, 424-426), and the
// planeStressWeakRes stack (:286-315): ADObj, SymMat, MatGreenStrain<LINEAR |
// NONLINEAR>, SymIsotropic, SymMatMultTrace, MakeStack(...).reverse().
//
// One deviation from a plain row-major matrix: a ONE-ROW Mat<T, 1, N> answers
// (i, j) with entry (0, j) for every i.  The reference's CPU Jacobian loop reads
// its one-row seed dudxDot as dudxDot(stateInd, jj) (FEKernels.h:460,469), past
// the end of the matrix for stateInd = 1, while its GPU kernel reads the same
// seed as dudxDot[jj] (FEKernels.h:936); with this rule the CPU loop reads what
// the GPU kernel reads instead of undefined memory.
//
// Conventions: Mat<T, M, N> is row-major, zero-initialised and converts to a
// pointer to its entries; zero() assigns
// T(0) to every entry (for ADScalar entries that clears the value and the
// derivatives).  SymMat<T, 2> stores (0,0), (0,1) = (1,0), (1,1); its seed
// (bvalue) holds the derivative with respect to each STORED entry, so an
// off-diagonal seed counts both (0,1) and (1,0).  MakeStack evaluates its
// expressions forward in argument order when it builds the stack (argument
// evaluation order is unspecified in C++, so the expressions only bind their
// operands); reverse() adds each one's contribution to its inputs' seeds, last
// expression first.
//
// TEST INFRASTRUCTURE ONLY: lets the reference's own CPU assembly compile as
// oracle/_ref (oracle/Makefile, target `ref`) so that the oracle restatement can
// be compared with it.  Nothing in the library under gpu-fem-project_b200/ uses it.
#pragma once

#include "adscalar.h"

namespace A2D {

enum class GreenStrainType { LINEAR, NONLINEAR };
enum class MatOp { NORMAL, TRANSPOSE };

template <typename T, int M, int N>
class Mat {
 public:
  T A[M * N];
  Mat() { zero(); }
  void zero() {
    for (int i = 0; i < M * N; i++) A[i] = T(0.0);
  }
  // A one-row matrix answers every row index with its row 0 (see the note above).
  T &operator()(int i, int j) { return A[(M == 1 ? 0 : N * i) + j]; }
  const T &operator()(int i, int j) const { return A[(M == 1 ? 0 : N * i) + j]; }
  T &operator[](int i) { return A[i]; }
  const T &operator[](int i) const { return A[i]; }
  T *get_data() { return A; }
  const T *get_data() const { return A; }
  // the reference passes matrices where its helpers take plain arrays
  // (e.g. FEKernels.h:354 -> :232, :371 -> :107)
  operator T *() { return A; }
  operator const T *() const { return A; }
};

template <typename T, int N>
class SymMat {
 public:
  static constexpr int SIZE = N * (N + 1) / 2;
  T A[SIZE];
  SymMat() { zero(); }
  void zero() {
    for (int i = 0; i < SIZE; i++) A[i] = T(0.0);
  }
  static int index(int i, int j) { return i >= j ? j + i * (i + 1) / 2 : i + j * (j + 1) / 2; }
  T &operator()(int i, int j) { return A[index(i, j)]; }
  const T &operator()(int i, int j) const { return A[index(i, j)]; }
};

// A value and its reverse-mode seed.
template <class T>
class ADObj {
 public:
  ADObj() : v(), b() {}
  ADObj(const T &x) : v(x), b() {}
  T &value() { return v; }
  const T &value() const { return v; }
  T &bvalue() { return b; }
  const T &bvalue() const { return b; }

 private:
  T v, b;
};

// C = op(A) op(B)
template <MatOp opA = MatOp::NORMAL, MatOp opB = MatOp::NORMAL, typename T, int AM, int AN, int BM, int BN, int CM,
          int CN>
void MatMatMult(const Mat<T, AM, AN> &A, const Mat<T, BM, BN> &B, Mat<T, CM, CN> &C) {
  constexpr int K = (opA == MatOp::NORMAL) ? AN : AM;
  static_assert(((opA == MatOp::NORMAL) ? AM : AN) == CM, "MatMatMult: row count");
  static_assert(((opB == MatOp::NORMAL) ? BN : BM) == CN, "MatMatMult: column count");
  static_assert(((opB == MatOp::NORMAL) ? BM : BN) == K, "MatMatMult: inner dimension");
  for (int i = 0; i < CM; i++) {
    for (int j = 0; j < CN; j++) {
      T s = T(0.0);
      for (int k = 0; k < K; k++) {
        const T a = (opA == MatOp::NORMAL) ? A(i, k) : A(k, i);
        const T b = (opB == MatOp::NORMAL) ? B(k, j) : B(j, k);
        s = s + a * b;
      }
      C(i, j) = s;
    }
  }
}

// 2x2 determinant and inverse (adjugate over the determinant).
template <typename T>
void MatDet(const Mat<T, 2, 2> &A, T &det) {
  det = A(0, 0) * A(1, 1) - A(0, 1) * A(1, 0);
}
template <typename T>
void MatInv(const Mat<T, 2, 2> &A, Mat<T, 2, 2> &Ainv) {
  const T det = A(0, 0) * A(1, 1) - A(0, 1) * A(1, 0);
  const T inv = T(1.0) / det;
  Ainv(0, 0) = A(1, 1) * inv;
  Ainv(0, 1) = -A(0, 1) * inv;
  Ainv(1, 0) = -A(1, 0) * inv;
  Ainv(1, 1) = A(0, 0) * inv;
}

// E = 1/2 (U + U^T) (LINEAR) or 1/2 (U + U^T + U^T U) (NONLINEAR), 2x2.
template <GreenStrainType type, typename T>
class MatGreenStrainExpr {
 public:
  MatGreenStrainExpr(ADObj<Mat<T, 2, 2>> &U, ADObj<SymMat<T, 2>> &E) : U(U), E(E) {}
  void eval() {
    const Mat<T, 2, 2> &u = U.value();
    SymMat<T, 2> &e = E.value();
    if constexpr (type == GreenStrainType::LINEAR) {
      e(0, 0) = u(0, 0);
      e(1, 1) = u(1, 1);
      e(0, 1) = T(0.5) * (u(0, 1) + u(1, 0));
    } else {
      e(0, 0) = u(0, 0) + T(0.5) * (u(0, 0) * u(0, 0) + u(1, 0) * u(1, 0));
      e(1, 1) = u(1, 1) + T(0.5) * (u(0, 1) * u(0, 1) + u(1, 1) * u(1, 1));
      e(0, 1) = T(0.5) * (u(0, 1) + u(1, 0) + u(0, 0) * u(0, 1) + u(1, 0) * u(1, 1));
    }
  }
  void reverse() {
    const Mat<T, 2, 2> &u = U.value();
    const SymMat<T, 2> &eb = E.bvalue();
    Mat<T, 2, 2> &ub = U.bvalue();
    const T h = T(0.5) * eb(0, 1);
    if constexpr (type == GreenStrainType::LINEAR) {
      ub(0, 0) = ub(0, 0) + eb(0, 0);
      ub(1, 1) = ub(1, 1) + eb(1, 1);
      ub(0, 1) = ub(0, 1) + h;
      ub(1, 0) = ub(1, 0) + h;
    } else {
      ub(0, 0) = ub(0, 0) + (eb(0, 0) * (T(1.0) + u(0, 0)) + h * u(0, 1));
      ub(1, 0) = ub(1, 0) + (eb(0, 0) * u(1, 0) + h * (T(1.0) + u(1, 1)));
      ub(0, 1) = ub(0, 1) + (eb(1, 1) * u(0, 1) + h * (T(1.0) + u(0, 0)));
      ub(1, 1) = ub(1, 1) + (eb(1, 1) * (T(1.0) + u(1, 1)) + h * u(1, 0));
    }
  }

 private:
  ADObj<Mat<T, 2, 2>> &U;
  ADObj<SymMat<T, 2>> &E;
};

template <GreenStrainType type, typename T>
MatGreenStrainExpr<type, T> MatGreenStrain(ADObj<Mat<T, 2, 2>> &U, ADObj<SymMat<T, 2>> &E) {
  return MatGreenStrainExpr<type, T>(U, E);
}

// S = 2 mu E + lambda tr(E) I
template <typename T>
class SymIsotropicExpr {
 public:
  SymIsotropicExpr(double mu, double lambda, ADObj<SymMat<T, 2>> &E, ADObj<SymMat<T, 2>> &S)
      : mu(mu), lambda(lambda), E(E), S(S) {}
  void eval() {
    const SymMat<T, 2> &e = E.value();
    SymMat<T, 2> &s = S.value();
    const T tr = e(0, 0) + e(1, 1);
    s(0, 0) = T(2.0 * mu) * e(0, 0) + T(lambda) * tr;
    s(1, 1) = T(2.0 * mu) * e(1, 1) + T(lambda) * tr;
    s(0, 1) = T(2.0 * mu) * e(0, 1);
  }
  void reverse() {
    const SymMat<T, 2> &sb = S.bvalue();
    SymMat<T, 2> &eb = E.bvalue();
    const T tr = sb(0, 0) + sb(1, 1);
    eb(0, 0) = eb(0, 0) + (T(2.0 * mu) * sb(0, 0) + T(lambda) * tr);
    eb(1, 1) = eb(1, 1) + (T(2.0 * mu) * sb(1, 1) + T(lambda) * tr);
    eb(0, 1) = eb(0, 1) + T(2.0 * mu) * sb(0, 1);
  }

 private:
  double mu, lambda;
  ADObj<SymMat<T, 2>> &E;
  ADObj<SymMat<T, 2>> &S;
};

template <typename T>
SymIsotropicExpr<T> SymIsotropic(double mu, double lambda, ADObj<SymMat<T, 2>> &E, ADObj<SymMat<T, 2>> &S) {
  return SymIsotropicExpr<T>(mu, lambda, E, S);
}

// out = sum_ij E_ij S_ij (the off-diagonal pair counted twice)
template <typename T>
class SymMatMultTraceExpr {
 public:
  SymMatMultTraceExpr(ADObj<SymMat<T, 2>> &E, ADObj<SymMat<T, 2>> &S, ADObj<T> &out) : E(E), S(S), out(out) {}
  void eval() {
    const SymMat<T, 2> &e = E.value(), &s = S.value();
    out.value() = e(0, 0) * s(0, 0) + e(1, 1) * s(1, 1) + T(2.0) * (e(0, 1) * s(0, 1));
  }
  void reverse() {
    const T ob = out.bvalue();
    const SymMat<T, 2> &e = E.value(), &s = S.value();
    SymMat<T, 2> &eb = E.bvalue(), &sb = S.bvalue();
    eb(0, 0) = eb(0, 0) + ob * s(0, 0);
    eb(1, 1) = eb(1, 1) + ob * s(1, 1);
    eb(0, 1) = eb(0, 1) + T(2.0) * (ob * s(0, 1));
    sb(0, 0) = sb(0, 0) + ob * e(0, 0);
    sb(1, 1) = sb(1, 1) + ob * e(1, 1);
    sb(0, 1) = sb(0, 1) + T(2.0) * (ob * e(0, 1));
  }

 private:
  ADObj<SymMat<T, 2>> &E;
  ADObj<SymMat<T, 2>> &S;
  ADObj<T> &out;
};

template <typename T>
SymMatMultTraceExpr<T> SymMatMultTrace(ADObj<SymMat<T, 2>> &E, ADObj<SymMat<T, 2>> &S, ADObj<T> &out) {
  return SymMatMultTraceExpr<T>(E, S, out);
}

// A sequence of expressions whose reverse() runs them last to first.
template <class... Exprs>
class Stack;
template <>
class Stack<> {
 public:
  void eval() {}
  void reverse() {}
};
template <class First, class... Rest>
class Stack<First, Rest...> {
 public:
  Stack(First f, Rest... r) : first(f), rest(r...) {}
  void eval() {
    first.eval();
    rest.eval();
  }
  void reverse() {
    rest.reverse();
    first.reverse();
  }

 private:
  First first;
  Stack<Rest...> rest;
};

template <class... Exprs>
Stack<Exprs...> MakeStack(Exprs... e) {
  Stack<Exprs...> s(e...);
  s.eval();
  return s;
}

}  // namespace A2D
