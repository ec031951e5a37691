// ============================================================================
// FP64 CPU ORACLE for plane-stress Lagrange-quad residual/Jacobian assembly.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: only tests/, the smoke
// check in __graft_entry__.py and the CPU-baseline leg of bench.py load it.  The
// product (the CUDA library under gpu-fem-project_b200/) never links or calls it.
//
// What it restates (file:line in A-CGray/GPU-FEM-Project):
//   * Gauss-Legendre points/weights, p+1 per direction ........ element/GaussQuadrature.h:47-100
//   * cosine-knot Lagrange basis values/derivatives (fma form,
//     the reference's own coefficient tables) ................. element/LagrangeShapeFuncs.h:7-10,129-216,244-252
//   * element gather ........................................... element/FEKernels.h:25-42
//   * isoparametric J, inverse, signed det ..................... element/FEKernels.h:230-257,352-359
//   * real-space state gradient ................................. element/FEKernels.h:260-284
//   * plane-stress weak residual (linear strain) ............... element/FEKernels.h:286-315
//   * residual transform (the "cost1 <= cost2" branch) ......... element/FEKernels.h:106-197
//   * residual assembly loop ................................... element/FEKernels.h:317-377
//   * Jacobian assembly, one forward-mode column at a time ...... element/FEKernels.h:379-508
//   * residual / BSR scatter .................................... element/FEKernels.h:44-104
//   * element -> BSR block map (linear search along a row) ..... verification/TACSHelpers.h:133-182
//
// The reference differentiates the strain energy with the A2D library, which is
// not vendored with the reference (no pinned version; only an include path at
// Makefile.in:2-3).  The restatement replaces that AD with the closed form it
// computes for GreenStrainType::LINEAR: weakRes = w*detJ*t*sigma, with
// sigma = 2*mu*eps + lambda*tr(eps)*I, mu = E/(2(1+nu)), lambda = 2*mu*nu/(1-nu),
// and the forward-mode Jacobian column is the same linear map applied to the
// seeded state gradient.  For GreenStrainType::NONLINEAR (a template option of
// the reference kernels, FEKernels.h:286,317,379,589,786, that its dispatch
// never selects) E = 1/2 (g + g^T + g^T g), S = 2 mu E + lambda tr(E) I,
// weakRes = w*detJ*t*(I + g) S, and the Jacobian column is its forward
// derivative along the seed, written out by hand (weakResDot).
//
// Pinning: the quadrature and shape-function tables are checked against the
// reference's own headers compiled from their source (oracle/_ref, recipe in
// oracle/Makefile).  The element physics is NOT pinned by reference outputs:
// the reference ships no fixtures and its A2D/TACS dependencies are absent, so
// the physics is checked by known-answer tests (analytic Q4 stiffness, rigid
// body modes, R = K u, finite differences, patch test) -- parity for the
// physics is "unpinned" in that sense.
//
// Two deliberate differences from the reference CPU path:
//   * the element matrix is stored row-major (row = DOF of the test function),
//     as the reference GPU kernel does (FEKernels.h:972-974); the reference CPU
//     loop stores its transpose (FEKernels.h:492), which is the same matrix
//     because Ke is symmetric for linear elasticity;
//   * the matrix scatter is race-free: elements are computed in parallel into
//     a chunk buffer and scattered serially in element order, so the oracle is
//     deterministic (the reference CPU scatter has no atomic, FEKernels.h:95-99).
// ============================================================================
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// element/GaussQuadrature.h:47-100 (orders 1..4, p+1 points).
const double kGaussX[5][5] = {
    {0.0, 0, 0, 0, 0},
    {-0.577350269189626, 0.577350269189626, 0, 0, 0},
    {-0.774596669241483, 0.0, 0.774596669241483, 0, 0},
    {-0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053, 0},
    {-0.906179845938664, -0.538469310105683, 0.0, 0.538469310105683, 0.906179845938664},
};
const double kGaussW[5][5] = {
    {2.0, 0, 0, 0, 0},
    {1.0, 1.0, 0, 0, 0},
    {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0, 0, 0},
    {0.347854845137454, 0.652145154862546, 0.652145154862546, 0.347854845137454, 0},
    {0.236926885056189, 0.478628670499366, 0.568888888888889, 0.478628670499366, 0.236926885056189},
};

// Monomial coefficients, highest power first (element/LagrangeShapeFuncs.h:131-216).
const double kC1[2][2] = {{-0.5, 0.5}, {0.5, 0.5}};
const double kC2[3][3] = {{0.5, -0.5, 0.0}, {-1.0, 0.0, 1.0}, {0.5, 0.5, 0.0}};
const double kC3[4][4] = {{-2.0 / 3.0, 2.0 / 3.0, 1.0 / 6.0, -1.0 / 6.0},
                          {4.0 / 3.0, -2.0 / 3.0, -4.0 / 3.0, 2.0 / 3.0},
                          {-4.0 / 3.0, -2.0 / 3.0, 4.0 / 3.0, 2.0 / 3.0},
                          {2.0 / 3.0, 2.0 / 3.0, -1.0 / 6.0, -1.0 / 6.0}};
const double kC4[5][5] = {{1.0, -1.0, -0.5, 0.5, 0.0},
                          {-2.0, 1.41421356237310, 2.0, -1.41421356237310, 0.0},
                          {2.0, 0.0, -3., 0.0, 1.0},
                          {-2.0, -1.41421356237310, 2.0, 1.41421356237310, 0.0},
                          {1.0, 1.0, -0.5, -0.5, 0.0}};

// lagrangePoly1dDeriv<double,p> (element/LagrangeShapeFuncs.h:129-216), same fma nesting.
inline void lagrange1d(int p, double x, int k, double &N, double &dN) {
  switch (p) {
    case 1: {
      const double *c = kC1[k];
      N = std::fma(c[0], x, c[1]);
      dN = c[0];
    } break;
    case 2: {
      const double *c = kC2[k];
      N = std::fma(c[0], x * x, std::fma(c[1], x, c[2]));
      dN = std::fma(2 * c[0], x, c[1]);
    } break;
    case 3: {
      const double *c = kC3[k];
      const double x2 = x * x, x3 = x2 * x;
      N = std::fma(c[0], x3, std::fma(c[1], x2, std::fma(c[2], x, c[3])));
      dN = std::fma(3 * c[0], x2, std::fma(2 * c[1], x, c[2]));
    } break;
    default: {
      const double *c = kC4[k];
      const double x2 = x * x, x3 = x2 * x, x4 = x2 * x2;
      N = std::fma(c[0], x4, std::fma(c[1], x3, std::fma(c[2], x2, std::fma(c[3], x, c[4]))));
      dN = std::fma(4 * c[0], x3, std::fma(3 * c[1], x2, std::fma(2 * c[2], x, c[3])));
    } break;
  }
}

// lagrangePoly2dDeriv (element/LagrangeShapeFuncs.h:244-252): [Ny*dNx, Nx*dNy].
inline void lagrange2dDeriv(int p, const double xi[2], int ax, int ay, double d[2]) {
  double Nx, dNx, Ny, dNy;
  lagrange1d(p, xi[0], ax, Nx, dNx);
  lagrange1d(p, xi[1], ay, Ny, dNy);
  d[0] = Ny * dNx;
  d[1] = Nx * dNy;
}

// strain: 0 = GreenStrainType::LINEAR (the reference's default), 1 = NONLINEAR.
struct Material {
  double mu, lambda, t;
  int strain;
};

inline Material makeMaterial(double E, double nu, double t, int strain = 0) {
  // element/FEKernels.h:300-301
  Material m;
  m.mu = 0.5 * E / (1.0 + nu);
  m.lambda = 2 * m.mu * nu / (1.0 - nu);
  m.t = t;
  m.strain = strain;
  return m;
}

// Green strain E = 1/2 (g + g^T + g^T g) (A2D MatGreenStrain<NONLINEAR>), stored
// [E00, E01, E11]; g[i*2+j] = du_i/dx_j.
inline void greenStrain(const double g[4], double e[3]) {
  e[0] = 0.5 * (2 * g[0] + g[0] * g[0] + g[2] * g[2]);
  e[1] = 0.5 * (g[1] + g[2] + g[0] * g[1] + g[2] * g[3]);
  e[2] = 0.5 * (2 * g[3] + g[1] * g[1] + g[3] * g[3]);
}

// Forward derivative of the Green strain along the seed gd.
inline void greenStrainDot(const double g[4], const double gd[4], double e[3]) {
  e[0] = 0.5 * (2 * gd[0] + 2 * (gd[0] * g[0] + gd[2] * g[2]));
  e[1] = 0.5 * (gd[1] + gd[2] + gd[0] * g[1] + g[0] * gd[1] + gd[2] * g[3] + g[2] * gd[3]);
  e[2] = 0.5 * (2 * gd[3] + 2 * (gd[1] * g[1] + gd[3] * g[3]));
}

// SymIsotropic: S = 2 mu E + lambda tr(E) I, [S00, S01, S11].
inline void isotropic(const Material &m, const double e[3], double s[3]) {
  const double tr = e[0] + e[2];
  s[0] = 2 * m.mu * e[0] + m.lambda * tr;
  s[1] = 2 * m.mu * e[1];
  s[2] = 2 * m.mu * e[2] + m.lambda * tr;
}

// planeStressWeakRes<strainType> closed form (element/FEKernels.h:286-315): the
// gradient of W = 1/2 scale t S:E with respect to g.
//   LINEAR:    E = sym(g), out = scale * t * sigma (symmetric).
//   NONLINEAR: E = 1/2 (g + g^T + g^T g), out = scale * t * (I + g) S.
inline void weakRes(const Material &m, double scale, const double g[4], double out[4]) {
  const double f = scale * m.t;
  if (m.strain == 0) {
    const double e00 = g[0], e11 = g[3], e01 = 0.5 * (g[1] + g[2]);
    const double tr = e00 + e11;
    const double s00 = 2 * m.mu * e00 + m.lambda * tr;
    const double s11 = 2 * m.mu * e11 + m.lambda * tr;
    const double s01 = 2 * m.mu * e01;
    out[0] = f * s00;
    out[1] = f * s01;
    out[2] = f * s01;
    out[3] = f * s11;
    return;
  }
  double e[3], S[3];
  greenStrain(g, e);
  isotropic(m, e, S);
  const double F00 = 1 + g[0], F01 = g[1], F10 = g[2], F11 = 1 + g[3];
  out[0] = f * (F00 * S[0] + F01 * S[1]);
  out[1] = f * (F00 * S[1] + F01 * S[2]);
  out[2] = f * (F10 * S[0] + F11 * S[1]);
  out[3] = f * (F10 * S[1] + F11 * S[2]);
}

// Forward-mode derivative of weakRes at g along the seed gd (the ADScalar<double,1>
// pass of element/FEKernels.h:444-472,926-940).  LINEAR: weakRes(gd).
//   NONLINEAR: scale * t * (gd S + (I + g) S'), S' = S(E'(g; gd)).
inline void weakResDot(const Material &m, double scale, const double g[4], const double gd[4], double out[4]) {
  if (m.strain == 0) {
    weakRes(m, scale, gd, out);
    return;
  }
  const double f = scale * m.t;
  double e[3], S[3], ed[3], Sd[3];
  greenStrain(g, e);
  isotropic(m, e, S);
  greenStrainDot(g, gd, ed);
  isotropic(m, ed, Sd);
  const double F00 = 1 + g[0], F01 = g[1], F10 = g[2], F11 = 1 + g[3];
  out[0] = f * (gd[0] * S[0] + gd[1] * S[1] + F00 * Sd[0] + F01 * Sd[1]);
  out[1] = f * (gd[0] * S[1] + gd[1] * S[2] + F00 * Sd[1] + F01 * Sd[2]);
  out[2] = f * (gd[2] * S[0] + gd[3] * S[1] + F10 * Sd[0] + F11 * Sd[1]);
  out[3] = f * (gd[2] * S[1] + gd[3] * S[2] + F10 * Sd[1] + F11 * Sd[2]);
}

// Strain energy density times scale * t: 1/2 scale t S:E (SymMatMultTrace).
inline double energy(const Material &m, double scale, const double g[4]) {
  double e[3], S[3];
  if (m.strain == 0) {
    e[0] = g[0];
    e[1] = 0.5 * (g[1] + g[2]);
    e[2] = g[3];
  } else {
    greenStrain(g, e);
  }
  isotropic(m, e, S);
  return 0.5 * scale * m.t * (S[0] * e[0] + 2 * S[1] * e[1] + S[2] * e[2]);
}

struct QuadPoint {
  double Jinv[4];
  double detJ;
  double scale;  // w * detJ
  double xi[2];
};

// Extended-precision mode (oracle_set_extended_j): J = sum_a x_a (x) dN_a is
// accumulated in long double (64-bit significand) and rounded to double once.  On
// large, finely divided meshes the FP64 sum cancels by ~h/|x| (the terms are ~|x|,
// J ~ h), so the plain sum carries an error of ~ulp(|x|)/|J| relative; the
// extended sum is the same formula on the same FP64 inputs, evaluated to ~1e-16.
bool g_extended_j = false;

// One quadrature point: J (interpParamGradient), MatInv/MatDet (FEKernels.h:352-359).
inline QuadPoint quadPoint(int p, int qx, int qy, const double *X) {
  QuadPoint Q;
  Q.xi[0] = kGaussX[p][qx];
  Q.xi[1] = kGaussX[p][qy];
  const double w = kGaussW[p][qx] * kGaussW[p][qy];
  double J[4] = {0, 0, 0, 0};
  long double JL[4] = {0, 0, 0, 0};
  for (int ay = 0; ay <= p; ay++) {
    for (int ax = 0; ax <= p; ax++) {
      const int a = ay * (p + 1) + ax;
      double d[2];
      lagrange2dDeriv(p, Q.xi, ax, ay, d);
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
          if (g_extended_j)
            JL[i * 2 + j] += (long double)X[a * 2 + i] * (long double)d[j];
          else
            J[i * 2 + j] += X[a * 2 + i] * d[j];
        }
    }
  }
  if (g_extended_j)
    for (int i = 0; i < 4; i++) J[i] = (double)JL[i];
  Q.detJ = J[0] * J[3] - J[1] * J[2];
  const double inv = 1.0 / Q.detJ;
  Q.Jinv[0] = J[3] * inv;
  Q.Jinv[1] = -J[1] * inv;
  Q.Jinv[2] = -J[2] * inv;
  Q.Jinv[3] = J[0] * inv;
  Q.scale = w * Q.detJ;
  return Q;
}

// interpRealGradient (FEKernels.h:260-284): dudx = (sum_a u_a (x) dN_a) * Jinv.
inline void realGradient(int p, const QuadPoint &Q, const double *U, double g[4]) {
  double gx[4] = {0, 0, 0, 0};
  for (int ay = 0; ay <= p; ay++) {
    for (int ax = 0; ax <= p; ax++) {
      const int a = ay * (p + 1) + ax;
      double d[2];
      lagrange2dDeriv(p, Q.xi, ax, ay, d);
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) gx[i * 2 + j] += U[a * 2 + i] * d[j];
    }
  }
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) g[i * 2 + j] = gx[i * 2 + 0] * Q.Jinv[0 * 2 + j] + gx[i * 2 + 1] * Q.Jinv[1 * 2 + j];
}

// addTransformStateGradSens, else-branch (FEKernels.h:170-196): temp = dN * Jinv,
// out(a,i) += sum_k temp(a,k) * W(i,k).
inline void transformAdd(int p, const QuadPoint &Q, const double W[4], double *out) {
  for (int ay = 0; ay <= p; ay++) {
    for (int ax = 0; ax <= p; ax++) {
      const int a = ay * (p + 1) + ax;
      double d[2];
      lagrange2dDeriv(p, Q.xi, ax, ay, d);
      double tmp[2] = {0, 0};
      for (int j = 0; j < 2; j++)
        for (int k = 0; k < 2; k++) tmp[j] += d[k] * Q.Jinv[k * 2 + j];
      for (int i = 0; i < 2; i++) out[a * 2 + i] += tmp[0] * W[i * 2 + 0] + tmp[1] * W[i * 2 + 1];
    }
  }
}

// gatherElementData (FEKernels.h:25-42).
inline void gather(int n, const int *connPtr, const int *conn, int64_t e, const double *states,
                   const double *coords, double *U, double *X) {
  for (int a = 0; a < n; a++) {
    const int node = conn[connPtr[e] + a];
    X[a * 2 + 0] = coords[(int64_t)node * 2 + 0];
    X[a * 2 + 1] = coords[(int64_t)node * 2 + 1];
    U[a * 2 + 0] = states[(int64_t)node * 2 + 0];
    U[a * 2 + 1] = states[(int64_t)node * 2 + 1];
  }
}

// Element residual and (optionally) element matrix, following the loop
// structure of assemblePlaneStressJacobian (FEKernels.h:379-508): quadrature x
// outer, y inner; per point the residual transform, then one forward column per
// nodal DOF (node y outer, x inner, state inner).
void elementKernel(int p, const double *X, const double *U, const Material &m, double *Re, double *Ke) {
  const int n = (p + 1) * (p + 1), nd = 2 * n;
  std::fill(Re, Re + nd, 0.0);
  if (Ke) std::fill(Ke, Ke + (size_t)nd * nd, 0.0);
  std::vector<double> col(nd);
  for (int qx = 0; qx <= p; qx++) {
    for (int qy = 0; qy <= p; qy++) {
      const QuadPoint Q = quadPoint(p, qx, qy, X);
      double g[4], W[4];
      realGradient(p, Q, U, g);
      weakRes(m, Q.scale, g, W);
      transformAdd(p, Q, W, Re);
      if (!Ke) continue;
      for (int by = 0; by <= p; by++) {
        for (int bx = 0; bx <= p; bx++) {
          const int b = by * (p + 1) + bx;
          double d[2];
          lagrange2dDeriv(p, Q.xi, bx, by, d);
          // dudxDot = dudxiDot * Jinv (FEKernels.h:462-463)
          const double gd0 = d[0] * Q.Jinv[0] + d[1] * Q.Jinv[2];
          const double gd1 = d[0] * Q.Jinv[1] + d[1] * Q.Jinv[3];
          for (int k = 0; k < 2; k++) {
            double seed[4] = {0, 0, 0, 0};
            seed[k * 2 + 0] = gd0;
            seed[k * 2 + 1] = gd1;
            double Wd[4];
            weakResDot(m, Q.scale, g, seed, Wd);
            std::fill(col.begin(), col.end(), 0.0);
            transformAdd(p, Q, Wd, col.data());
            const int c = b * 2 + k;
            for (int r = 0; r < nd; r++) Ke[(size_t)r * nd + c] += col[r];
          }
        }
      }
    }
  }
}

}  // namespace

extern "C" {

int oracle_version() { return 1; }

// 1: accumulate the isoparametric Jacobian in long double (see g_extended_j);
// 0: the reference's plain FP64 sum (default).
void oracle_set_extended_j(int on) { g_extended_j = on != 0; }

int oracle_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// Gauss points/weights (1D, p+1 each) and the 2D derivative table
// dN[q][a][2], q = qy*(p+1)+qx, a = ay*(p+1)+ax.
int oracle_tables(int p, double *xi, double *w, double *dN) {
  if (p < 1 || p > 4) return 1;
  for (int i = 0; i <= p; i++) {
    xi[i] = kGaussX[p][i];
    w[i] = kGaussW[p][i];
  }
  const int n = (p + 1) * (p + 1);
  for (int qy = 0; qy <= p; qy++)
    for (int qx = 0; qx <= p; qx++) {
      const double x[2] = {kGaussX[p][qx], kGaussX[p][qy]};
      const int q = qy * (p + 1) + qx;
      for (int ay = 0; ay <= p; ay++)
        for (int ax = 0; ax <= p; ax++) {
          const int a = ay * (p + 1) + ax;
          lagrange2dDeriv(p, x, ax, ay, &dN[((size_t)q * n + a) * 2]);
        }
    }
  return 0;
}

// 1D basis value/derivative at arbitrary points, for table and partition-of-unity checks.
int oracle_lagrange1d(int p, int npts, const double *x, double *N, double *dN) {
  if (p < 1 || p > 4) return 1;
  for (int i = 0; i < npts; i++)
    for (int k = 0; k <= p; k++) lagrange1d(p, x[i], k, N[i * (p + 1) + k], dN[i * (p + 1) + k]);
  return 0;
}

// One element: Re[2n] and Ke[2n*2n] (row-major, DOF = node*2 + state).
// strain: 0 = LINEAR, 1 = NONLINEAR Green strain.
int oracle_element_ex(int p, const double *X, const double *U, double E, double nu, double t, int strain, double *Re,
                      double *Ke) {
  if (p < 1 || p > 4 || strain < 0 || strain > 1) return 1;
  elementKernel(p, X, U, makeMaterial(E, nu, t, strain), Re, Ke);
  return 0;
}

int oracle_element(int p, const double *X, const double *U, double E, double nu, double t, double *Re, double *Ke) {
  return oracle_element_ex(p, X, U, E, nu, t, 0, Re, Ke);
}

// Element strain energy sum_q 1/2 w detJ t S:E (the quantity the reference's
// weak residual differentiates), for finite-difference checks of the residual.
int oracle_element_energy(int p, const double *X, const double *U, double E, double nu, double t, int strain,
                          double *W) {
  if (p < 1 || p > 4 || strain < 0 || strain > 1) return 1;
  const Material m = makeMaterial(E, nu, t, strain);
  double sum = 0;
  for (int qx = 0; qx <= p; qx++)
    for (int qy = 0; qy <= p; qy++) {
      const QuadPoint Q = quadPoint(p, qx, qy, X);
      double g[4];
      realGradient(p, Q, U, g);
      sum += energy(m, Q.scale, g);
    }
  *W = sum;
  return 0;
}

// assemblePlaneStressResidual / assemblePlaneStressJacobian (FEKernels.h:317-508)
// with the runJacobianKernel contract (FEKernels.h:1125-1136): accumulate into
// residual (nullable) and matEntries (nullable); map[e*n*n + a*n + b] is the
// offset (in doubles) of the 2x2 block coupling local nodes a and b.
int oracle_assemble_ex(int p, const int *connPtr, const int *conn, int64_t numElements, const double *states,
                       const double *coords, double E, double nu, double t, int strain, const int *map,
                       double *residual, double *matEntries) {
  if (p < 1 || p > 4 || strain < 0 || strain > 1) return 1;
  const int n = (p + 1) * (p + 1), nd = 2 * n;
  const Material m = makeMaterial(E, nu, t, strain);
  const bool jac = (matEntries != nullptr && map != nullptr);
  const int64_t chunk = 4096;
  std::vector<double> reBuf((size_t)chunk * nd);
  std::vector<double> keBuf(jac ? (size_t)chunk * nd * nd : 0);
  for (int64_t e0 = 0; e0 < numElements; e0 += chunk) {
    const int64_t ne = std::min(chunk, numElements - e0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < ne; i++) {
      double X[50], U[50];
      gather(n, connPtr, conn, e0 + i, states, coords, U, X);
      elementKernel(p, X, U, m, &reBuf[(size_t)i * nd], jac ? &keBuf[(size_t)i * nd * nd] : nullptr);
    }
    for (int64_t i = 0; i < ne; i++) {
      const int64_t e = e0 + i;
      const int *en = &conn[connPtr[e]];
      if (residual) {
        // scatterResidual (FEKernels.h:44-61)
        for (int a = 0; a < n; a++)
          for (int s = 0; s < 2; s++) residual[(int64_t)en[a] * 2 + s] += reBuf[(size_t)i * nd + a * 2 + s];
      }
      if (jac) {
        // scatterMat (FEKernels.h:63-104)
        const double *K = &keBuf[(size_t)i * nd * nd];
        const int *em = &map[e * n * n];
        for (int a = 0; a < n; a++)
          for (int b = 0; b < n; b++) {
            double *blk = &matEntries[em[a * n + b]];
            for (int ii = 0; ii < 2; ii++)
              for (int jj = 0; jj < 2; jj++) blk[ii * 2 + jj] += K[(size_t)(a * 2 + ii) * nd + b * 2 + jj];
          }
      }
    }
  }
  return 0;
}

int oracle_assemble(int p, const int *connPtr, const int *conn, int64_t numElements, const double *states,
                    const double *coords, double E, double nu, double t, const int *map, double *residual,
                    double *matEntries) {
  return oracle_assemble_ex(p, connPtr, conn, numElements, states, coords, E, nu, t, 0, map, residual, matEntries);
}

// Throughput variant used as the timed CPU baseline: OpenMP over elements with
// atomic scatters, like the reference CPU path (FEKernels.h:328,392) but with
// the matrix scatter made atomic.  Non-deterministic summation order.
int oracle_assemble_parallel(int p, const int *connPtr, const int *conn, int64_t numElements,
                             const double *states, const double *coords, double E, double nu, double t,
                             const int *map, double *residual, double *matEntries) {
  if (p < 1 || p > 4) return 1;
  const int n = (p + 1) * (p + 1), nd = 2 * n;
  const Material m = makeMaterial(E, nu, t);
  const bool jac = (matEntries != nullptr && map != nullptr);
#pragma omp parallel
  {
    std::vector<double> Re(nd), Ke(jac ? (size_t)nd * nd : 0);
#pragma omp for schedule(dynamic, 64)
    for (int64_t e = 0; e < numElements; e++) {
      double X[50], U[50];
      gather(n, connPtr, conn, e, states, coords, U, X);
      elementKernel(p, X, U, m, Re.data(), jac ? Ke.data() : nullptr);
      const int *en = &conn[connPtr[e]];
      if (residual)
        for (int a = 0; a < n; a++)
          for (int s = 0; s < 2; s++) {
#pragma omp atomic
            residual[(int64_t)en[a] * 2 + s] += Re[a * 2 + s];
          }
      if (jac) {
        const int *em = &map[e * n * n];
        for (int a = 0; a < n; a++)
          for (int b = 0; b < n; b++) {
            double *blk = &matEntries[em[a * n + b]];
            for (int ii = 0; ii < 2; ii++)
              for (int jj = 0; jj < 2; jj++) {
#pragma omp atomic
                blk[ii * 2 + jj] += Ke[(size_t)(a * 2 + ii) * nd + b * 2 + jj];
              }
          }
      }
    }
  }
  return 0;
}

// BSR sparsity of the nodal adjacency (the pattern TACS builds for the
// reference driver, TestKernels.cpp:105-115): row r holds every node that
// shares an element with node r, itself included, sorted ascending.  Written
// independently of the product's builder (per-row std::vector + sort/unique).
// Call with cols == nullptr to get nnzb only.
int64_t oracle_bsr_pattern(int numNodes, const int *connPtr, const int *conn, int64_t numElements, int *rowp,
                           int *cols) {
  std::vector<std::vector<int>> rows(numNodes);
  for (int64_t e = 0; e < numElements; e++) {
    const int b0 = connPtr[e], b1 = connPtr[e + 1];
    for (int i = b0; i < b1; i++)
      for (int j = b0; j < b1; j++) rows[conn[i]].push_back(conn[j]);
  }
  int64_t nnz = 0;
  for (int r = 0; r < numNodes; r++) {
    auto &v = rows[r];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    if (rowp) rowp[r] = (int)nnz;
    if (cols) std::copy(v.begin(), v.end(), cols + nnz);
    nnz += (int64_t)v.size();
  }
  if (rowp) rowp[numNodes] = (int)nnz;
  return nnz;
}

// generateElementBCSRMap (verification/TACSHelpers.h:138-182): linear search
// along row conn[a] for column conn[b]; value = block index * bsize^2 (bsize 2).
// Returns the number of blocks that were not found (0 on success).
int64_t oracle_element_bsr_map(const int *connPtr, const int *conn, int64_t numElements, int nodesPerElement,
                               const int *rowp, const int *cols, int *map) {
  const int n = nodesPerElement;
  int64_t missing = 0;
  for (int64_t e = 0; e < numElements; e++) {
    const int *en = &conn[connPtr[e]];
    for (int a = 0; a < n; a++) {
      const int r = en[a];
      for (int b = 0; b < n; b++) {
        bool found = false;
        for (int64_t jj = rowp[r]; jj < rowp[r + 1]; jj++) {
          if (cols[jj] == en[b]) {
            map[e * n * n + a * n + b] = (int)(jj * 4);
            found = true;
            break;
          }
        }
        if (!found) missing++;
      }
    }
  }
  return missing;
}

// Colouring validity: no two elements of one colour share a node.  Returns the
// number of conflicting (node, colour) pairs.
int64_t oracle_check_colouring(int numNodes, const int *connPtr, const int *conn, int64_t numElements,
                               const int *colour, int numColours) {
  std::vector<int64_t> last((size_t)numNodes * numColours, -1);
  int64_t bad = 0;
  for (int64_t e = 0; e < numElements; e++) {
    const int c = colour[e];
    if (c < 0 || c >= numColours) {
      bad++;
      continue;
    }
    for (int i = connPtr[e]; i < connPtr[e + 1]; i++) {
      int64_t &slot = last[(size_t)conn[i] * numColours + c];
      if (slot >= 0 && slot != e) bad++;
      slot = e;
    }
  }
  return bad;
}

// y = A x for a 2x2-block BSR matrix (used for the R = K u identity).
void oracle_bsr_spmv(int numRows, const int *rowp, const int *cols, const double *A, const double *x, double *y) {
#pragma omp parallel for schedule(static)
  for (int r = 0; r < numRows; r++) {
    double y0 = 0, y1 = 0;
    for (int64_t j = rowp[r]; j < rowp[r + 1]; j++) {
      const double *b = &A[j * 4];
      const double x0 = x[(int64_t)cols[j] * 2], x1 = x[(int64_t)cols[j] * 2 + 1];
      y0 += b[0] * x0 + b[1] * x1;
      y1 += b[2] * x0 + b[3] * x1;
    }
    y[(int64_t)r * 2] = y0;
    y[(int64_t)r * 2 + 1] = y1;
  }
}

}  // extern "C"
