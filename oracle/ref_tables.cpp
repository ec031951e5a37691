// Dumps the quadrature and shape-derivative tables computed by the reference's
// own headers (element/GaussQuadrature.h, element/LagrangeShapeFuncs.h), so the
// oracle's restated tables can be pinned against them bit for bit.
// Output: one line per value, "%a" (exact hexadecimal float).
#include <cstdio>

#include "GPUMacros.h"
#include "GaussQuadrature.h"
#include "LagrangeShapeFuncs.h"

template <int p>
void dump() {
  for (int i = 0; i <= p; i++) printf("gauss %d %d %a %a\n", p, i, getGaussQuadCoord<p>(i), getGaussQuadWeight<p>(i));
  for (int qy = 0; qy <= p; qy++)
    for (int qx = 0; qx <= p; qx++) {
      const double xi[2] = {getGaussQuadCoord<p>(qx), getGaussQuadCoord<p>(qy)};
      for (int ay = 0; ay <= p; ay++)
        for (int ax = 0; ax <= p; ax++) {
          double N = 0.0, d[2];
          lagrangePoly2dDeriv<double, p>(xi, ax, ay, N, d);
          printf("dN %d %d %d %a %a\n", p, qy * (p + 1) + qx, ay * (p + 1) + ax, d[0], d[1]);
        }
    }
  // 1D values/derivatives at a few fixed points
  const double xs[5] = {-1.0, -0.3, 0.0, 0.45, 1.0};
  for (int i = 0; i < 5; i++)
    for (int k = 0; k <= p; k++) {
      double N, dN;
      lagrangePoly1dDeriv<double, p>(xs[i], k, N, dN);
      printf("N1d %d %d %d %a %a %a\n", p, i, k, xs[i], N, dN);
    }
}

int main() {
  dump<1>();
  dump<2>();
  dump<3>();
  dump<4>();
  return 0;
}
