// Element assembly kernels for plane-stress Lagrange quads (orders 1..4) on sm_100a.
//
// One CTA processes EPB elements per step of a grid-stride loop (persistent
// grid sized from the occupancy of the instantiation):
//   1. gather      node ids, coordinates and states of the EPB elements
//                  (double2 loads through the read-only path) into shared memory;
//   2. quad points one thread per (element, q): J, signed detJ, J^-1, the
//                  real-space state gradient and the weak stress
//                  S = w*detJ*t*sigma (FP64 always);
//   3. gradients   one thread per (element, q, node): G = dN*J^-1 and the
//                  scaled copy H = w*detJ*t*G in the element arithmetic type T;
//   4. residual    one thread per (element, node): R_a = sum_q S G_a;
//   5. stiffness   one thread per (element, row tile of p+1 nodes, column node b):
//                  M_ij[a][b] = sum_q H_ai G_bj for the p+1 rows a of the tile,
//                  then the 2x2 block
//                    K_xx = (lam+2mu) M_xx + mu M_yy,  K_xy = lam M_xy + mu M_yx,
//                    K_yx = lam M_yx + mu M_xy,        K_yy = (lam+2mu) M_yy + mu M_xx.
// That is the closed form of the reference's per-column forward AD through
// planeStressWeakRes (element/FEKernels.h:286-315, 884-976): the seed of DOF
// (b,k) gives weakResDot = w detJ t sigma(e_k (x) G_b), and its transform onto
// DOF (a,i) is Ke[(a,i),(b,k)] = lam' M_ik + mu M_ki + mu delta_ik (M_xx + M_yy).
//
// Scatter: the drop-in mode adds through the reference's element->block map with
// FP64 atomics (element/FEKernels.h:730-780).  The plan mode runs one colour per
// launch; the first contributor to a block writes it with one 256-bit store (no
// zeroing, no read), later colours add with fire-and-forget reductions, and no
// two elements of one colour touch the same block or residual row.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "fem_umma.cuh"

namespace fem {
namespace dev {

// Gauss-Legendre points/weights (element/GaussQuadrature.h:47-100), p+1 per direction.
__constant__ double kGX[5][5] = {
    {0.0, 0, 0, 0, 0},
    {-0.577350269189626, 0.577350269189626, 0, 0, 0},
    {-0.774596669241483, 0.0, 0.774596669241483, 0, 0},
    {-0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053, 0},
    {-0.906179845938664, -0.538469310105683, 0.0, 0.538469310105683, 0.906179845938664},
};
__constant__ double kGW[5][5] = {
    {2.0, 0, 0, 0, 0},
    {1.0, 1.0, 0, 0, 0},
    {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0, 0, 0},
    {0.347854845137454, 0.652145154862546, 0.652145154862546, 0.347854845137454, 0},
    {0.236926885056189, 0.478628670499366, 0.568888888888889, 0.478628670499366, 0.236926885056189},
};
// Cosine-knot Lagrange monomial coefficients, highest power first
// (element/LagrangeShapeFuncs.h:131-216), [order][node][coefficient].
__constant__ double kCoef[5][5][5] = {
    {{0}},
    {{-0.5, 0.5}, {0.5, 0.5}},
    {{0.5, -0.5, 0.0}, {-1.0, 0.0, 1.0}, {0.5, 0.5, 0.0}},
    {{-2.0 / 3.0, 2.0 / 3.0, 1.0 / 6.0, -1.0 / 6.0},
     {4.0 / 3.0, -2.0 / 3.0, -4.0 / 3.0, 2.0 / 3.0},
     {-4.0 / 3.0, -2.0 / 3.0, 4.0 / 3.0, 2.0 / 3.0},
     {2.0 / 3.0, 2.0 / 3.0, -1.0 / 6.0, -1.0 / 6.0}},
    {{1.0, -1.0, -0.5, 0.5, 0.0},
     {-2.0, 1.41421356237310, 2.0, -1.41421356237310, 0.0},
     {2.0, 0.0, -3., 0.0, 1.0},
     {-2.0, -1.41421356237310, 2.0, 1.41421356237310, 0.0},
     {1.0, 1.0, -0.5, -0.5, 0.0}},
};

// lagrangePoly1dDeriv<double,p> (element/LagrangeShapeFuncs.h:129-216) with the
// rounding of every step pinned, so the table matches the host restatement bit for bit.
__device__ __forceinline__ void lag1d(int p, double x, int k, double &N, double &dN) {
  const double *c = kCoef[p][k];
  if (p == 1) {
    N = __fma_rn(c[0], x, c[1]);
    dN = c[0];
  } else if (p == 2) {
    N = __fma_rn(c[0], __dmul_rn(x, x), __fma_rn(c[1], x, c[2]));
    dN = __fma_rn(__dmul_rn(2.0, c[0]), x, c[1]);
  } else if (p == 3) {
    const double x2 = __dmul_rn(x, x), x3 = __dmul_rn(x2, x);
    N = __fma_rn(c[0], x3, __fma_rn(c[1], x2, __fma_rn(c[2], x, c[3])));
    dN = __fma_rn(__dmul_rn(3.0, c[0]), x2, __fma_rn(__dmul_rn(2.0, c[1]), x, c[2]));
  } else {
    const double x2 = __dmul_rn(x, x), x3 = __dmul_rn(x2, x), x4 = __dmul_rn(x2, x2);
    N = __fma_rn(c[0], x4, __fma_rn(c[1], x3, __fma_rn(c[2], x2, __fma_rn(c[3], x, c[4]))));
    dN = __fma_rn(__dmul_rn(4.0, c[0]), x3,
                  __fma_rn(__dmul_rn(3.0, c[1]), x2, __fma_rn(__dmul_rn(2.0, c[2]), x, c[3])));
  }
}

// One 2x2 block (32 bytes, 32-byte aligned) with a single 256-bit store.
__device__ __forceinline__ void store_block(double *p, double a, double b, double c, double d) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a), "d"(b), "d"(c), "d"(d) : "memory");
}

template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
  using type = double2;
};
template <>
struct Vec2<float> {
  using type = float2;
};

// kNL: GreenStrainType::NONLINEAR (Green strain, FP64 only); default LINEAR.
// kB16: fragment kernel, element stiffness on BF16 tensor cores with three-way split
// operands (FEM_PRECISION_MIXED at orders 2 and 3).
// kU: element kernel (order 4, FP32 element arithmetic), element stiffness as BF16x6
// products on the fifth-generation tensor cores (tcgen05, accumulator in TMEM).
enum : int { kRes = 1, kJac = 2, kPlan = 4, kNL = 8, kB16 = 32, kU = 64 };

struct AsmArgs {
  // drop-in fields | order-1 plan row tables (a plan never reads the drop-in ones)
  union {
    const int *connPtr;     // drop-in: CSR offsets
    const int *rowElemPtr;  // plan, order 1: per row, range of rowElem entries
  };
  union {
    const int *conn;     // drop-in: node ids
    const int *rowElem;  // plan, order 1: {k << 2 | a, four ranks} per (row, element)
  };
  union {
    const int *map;       // drop-in: element block offsets (doubles)
    const int *rowChunk;  // plan, order 1: row ranges of the warp chunks
  };
  const int *connList;       // plan: node ids of the listed elements, nn each
  const uint8_t *blockCode;  // plan: per listed element a Dims<P>::CS-byte code record
  const int *rowp;           // plan: BSR row pointers
  const double *states;
  const double *coords;
  double *residual;
  double *mat;
  double mu, lam, t;
  int64_t begin, count;  // element (or list position, or row chunk) range of this launch
  int *waits;            // plan: count of bounded in-kernel waits that ran out (nullptr: not counted)
};

// The output side of one batch: global outputs (registers) and the batch's
// staged block codes / element map in shared memory.
struct Out {
  double *mat;
  double *residual;
  const uint8_t *codes;  // plan: code records of the batch's elements (shared memory)
  const int *rbase;      // plan: rowp[node] per (element, node) (shared memory)
  const int *map;        // drop-in: element map rows of the batch (shared memory)
};

// Asynchronous global -> shared copies (no registers held while in flight).
__device__ __forceinline__ void cp_async16(void *sdst, const void *gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async4(void *sdst, const void *gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__host__ __device__ constexpr size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Launch shape per order: GT threads per group, EPG elements per group step,
// GPC independent groups per CTA (each synchronises on its own named barrier),
// NPART threads per quadrature point in the Jacobian stage, MINB resident CTAs
// per SM the register budget is sized for.  Stiffness-stage threads per element:
// the (p+1)-row tiles on or above the diagonal, 6 / 18 / 40 / 75 for p = 1..4.
template <int P>
struct Shape;
template <>
struct Shape<1> {
  static constexpr int GT = 64, EPG = 8, GPC = 4, NPART = 2, MINB = 3;
};
template <>
struct Shape<2> {
  static constexpr int GT = 64, EPG = 2, GPC = 4, NPART = 2, MINB = 3;
};
template <>
struct Shape<3> {
  static constexpr int GT = 64, EPG = 2, GPC = 2, NPART = 2, MINB = 5;
};
template <>
struct Shape<4> {
  static constexpr int GT = 128, EPG = 1, GPC = 1, NPART = 4, MINB = 4;
};

// Warps that share one element's stiffness MMA and the tile rows [R[w], R[w+1])
// each takes (p = 4: 7 + 6 + 9 + 6 of the 28 upper tiles of the 7x7 tile grid).
template <int P>
struct RowSplit {
  static constexpr int WPE = 1;
};
template <>
struct RowSplit<3> {
  static constexpr int WPE = 2;
};
template <>
struct RowSplit<4> {
  static constexpr int WPE = 4;
};

// Launch shape of the NONLINEAR kernels: four lanes per quadrature point in the
// quadrature stage (their shared-memory stores then hit 16 distinct banks).
template <int P>
struct NLShape;
template <>
struct NLShape<1> {
  static constexpr int GT = 64, EPG = 8, GPC = 2, NPART = 4, MINB = 3;
};
template <>
struct NLShape<2> {
  static constexpr int GT = 64, EPG = 2, GPC = 2, NPART = 4, MINB = 3;
};
template <>
struct NLShape<3> {
  static constexpr int GT = 64, EPG = 2, GPC = 2, NPART = 4, MINB = 3;
};
template <>
struct NLShape<4> {
  static constexpr int GT = 128, EPG = 1, GPC = 1, NPART = 4, MINB = 3;
};
template <int P, int MODE>
using ShapeSel = typename std::conditional<(MODE & kNL) != 0, NLShape<P>, Shape<P>>::type;

// NONLINEAR stiffness geometry.  With Phi the map from nodal DOFs to the state
// gradient and A the tangent modulus d2W/dg2 (4x4, g = du/dx),
//   K[(a,i),(b,k)] = sum_q s sum_{l,n} G_al A_{il,kn} G_bn,
// a product over kappa = (l, q) of the gradient array GA[kappa][a] = G-hat_al
// and GB[kappa][(2i+k)*NP + b] = sign(s) sum_n A_{il,kn} G-hat_bn (G-hat =
// sqrt|s| G).  Nodes are padded to NP (multiple of 8, m8n8k4 tiles of NTN node
// tiles), kappa to KN (multiple of 4).  Row strides RA, RB are 4 (mod 16) doubles:
// the four kappa rows of a fragment load and the four quadrature points of a
// quadrature-stage store cover 16 distinct banks.
template <int P>
struct NLDims {
  static constexpr int NN = (P + 1) * (P + 1), NQ = NN;
  static constexpr int NP = (NN + 7) / 8 * 8, NTN = NP / 8, NPAIR = NTN * (NTN + 1) / 2;
  static constexpr int KN = (2 * NQ + 3) / 4 * 4, KSN = KN / 4;
  static constexpr int RA = NP + 4, RB = 4 * NP + 4;
};

template <int P>
struct Dims {
  static constexpr int P1 = P + 1, NN = P1 * P1, NQ = NN;
  // upper-triangle row tiles: row tile `at` covers nodes at*P1 .. at*P1+P, columns b >= at*P1
  static constexpr int NTILE = P1 * NN - P1 * P1 * (P1 - 1) / 2;
  // FP64 tensor-core (m8n8k4) geometry of M = H^T G: rows/cols r = 2*node + component
  // padded to NT8 tiles of 8, the quadrature (k) dimension padded to NQP = 4*KS,
  // shared-memory row stride RS doubles with RS = 4 or 12 (mod 16): the four
  // quadrature rows of a fragment load then cover every bank exactly twice, and
  // the 16-byte gradient stores of the quadrature stage spread over all 8 bank groups.
  static constexpr int NT8 = (2 * NN + 7) / 8;
  static constexpr int KS = (NQ + 3) / 4, NQP = 4 * KS;
  static constexpr int RS = 8 * NT8 + 4;  // 8*NT8 is 0 or 8 mod 16
  // plan code record per element: NN*NN block codes + NN node codes, 16-byte padded
  static constexpr int CS = (NN * NN + NN + 15) / 16 * 16;
};

// Shared memory: per-CTA table, then GPC group regions.
//   FP64 (tensor-core stiffness): G and H as [NQP][RS] doubles, row r = 2a + i.
//   FP32 (CUDA-core stiffness):   G and H as [NQ][NN+1] float2, the padded row
//   lets the quadrature stage store without bank conflicts.
template <int P, typename T, int MODE>
struct Layout {
  using S = ShapeSel<P, MODE>;
  using D = Dims<P>;
  using ND = NLDims<P>;
  static constexpr bool TC = sizeof(T) == 8;
  static constexpr bool NL = (MODE & kNL) != 0;
  static_assert(!NL || TC, "NONLINEAR strain runs in FP64");
  static constexpr int NN = D::NN, NQ = NN, NNP = NN + 1, EPG = S::EPG;
  // FP64: one scaled-gradient array per element (G-hat, below); FP32: G and H;
  // NONLINEAR: GA then GB
  static constexpr size_t GA_ELEM = 8 * ND::KN * ND::RA;
  static constexpr size_t GH_ELEM = NL   ? GA_ELEM + 8 * ND::KN * ND::RB
                                    : TC ? 8 * D::NQP * D::RS
                                         : 2 * sizeof(T) * NQ * NNP;  // bytes per element
  static constexpr size_t H_ELEM = TC ? 0 : GH_ELEM;
  static constexpr int NSTRESS = NL ? 4 : 3;  // weak stress components (first Piola: 4)
  static constexpr size_t tabT = 0;                     // double2 [NN][NQ]
  static constexpr size_t wq = tabT + 16 * NQ * NN;     // double  [NQ]
  static constexpr size_t csum = align16(wq + 8 * NQ);  // double2 [NQ]: sum_a dN(a, q)
  static constexpr size_t groups = align16(csum + 16 * NQ);
  // group-relative
  static constexpr size_t X = 0;                               // double2 [EPG][NN]
  static constexpr size_t U = X + 16 * EPG * NN;               // double2 [EPG][NN]
  static constexpr size_t S3 = U + 16 * EPG * NN;  // double [NSTRESS][EPG*NQ] weak stress (SoA)
  static constexpr size_t G = align16(S3 + 8 * NSTRESS * EPG * NQ);  // [EPG] x GH_ELEM
  static constexpr size_t H = align16(G + EPG * GH_ELEM);            // [EPG] x H_ELEM
  static constexpr size_t SG = align16(H + EPG * H_ELEM);  // double [EPG][NQP]: sign of w detJ t (FP64 linear)
  static constexpr size_t nid = align16(SG + (TC && !NL ? 8 * EPG * D::NQP : 0));  // int [EPG][NN]
  static constexpr size_t rbase = align16(nid + 4 * EPG * NN);  // int [EPG][NN]
  // staged code records (plan) or element map rows (drop-in Jacobian), double-buffered
  static constexpr size_t STAGE = (MODE & kPlan) ? size_t(EPG) * D::CS
                                  : (MODE & kJac) ? size_t(EPG) * NN * NN * 4
                                                  : 16;
  static constexpr size_t stage = align16(rbase + 4 * EPG * NN);  // [2][STAGE] bytes
  static constexpr size_t group_bytes = align16(stage + 2 * align16(STAGE));
  // kU: BF16 operand tiles [A, B][part hi, mid, lo][K-step 0, 1] (umma::kTileBytes
  // each), the MMA-completion mbarrier and the TMEM base address
  static constexpr bool UM = (MODE & kU) != 0;
  static_assert(!UM || (P == 4 && !TC && !NL && S::GPC == 1 && S::EPG == 1 && S::GT == 128),
                "tcgen05 stiffness: order 4, FP32 element arithmetic, one 128-thread group per CTA");
  static constexpr size_t uop = (groups + S::GPC * group_bytes + 127) & ~size_t(127);
  static constexpr size_t umbar = uop + (UM ? 12 * umma::kTileBytes : 0);
  static constexpr size_t utmem = umbar + 8;
  static constexpr size_t total = UM ? utmem + 8 : groups + S::GPC * group_bytes;
};

__device__ __forceinline__ void group_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Writes the element block K(a,b) (and K(b,a) = K(a,b)^T when a != b) through the
// plan codes or the reference map.  `which`: 0 = block (a,b), 1 = block (b,a).
template <int P, int MODE>
__device__ __forceinline__ void write_block(const Out &A, int el, int a, int b, int which, double kxx, double kxy,
                                            double kyx, double kyy) {
  constexpr int NN = Dims<P>::NN, CS = Dims<P>::CS;
  const int r0 = which ? b : a, c0 = which ? a : b;
  const double v0 = kxx, v1 = which ? kyx : kxy, v2 = which ? kxy : kyx, v3 = kyy;
  if constexpr ((MODE & kPlan) != 0) {
    const uint8_t code = A.codes[el * CS + r0 * NN + c0];
    double *blk = A.mat + 4 * ((int64_t)A.rbase[el * NN + r0] + (code & 0x7f));
    if (code & 0x80) {
      store_block(blk, v0, v1, v2, v3);
    } else {
      // later colour: the first contributor's store is complete (previous launch)
      // and no element of this colour shares the block
      atomicAdd(blk + 0, v0);
      atomicAdd(blk + 1, v1);
      atomicAdd(blk + 2, v2);
      atomicAdd(blk + 3, v3);
    }
  } else {
    double *blk = A.mat + A.map[(el * NN + r0) * NN + c0];
    atomicAdd(blk + 0, v0);
    atomicAdd(blk + 1, v1);
    atomicAdd(blk + 2, v2);
    atomicAdd(blk + 3, v3);
  }
}

// One warp, tile rows [R0, R1) of the upper triangle of M = H^T G (FP64 MMA),
// then the 2x2 stiffness blocks.  Lane l holds C[8ti + l/4][8tj + 2(l%4) + {0,1}]
// = (M_i0, M_i1)[a][b] with a = (8ti + l/4)/2, i = (l/4)%2, b = 4tj + l%4; the
// lane with the other i (l ^ 4) supplies the second row of the block.
// M = H^T G with H = s G (s = w detJ t per quadrature point) is formed from the
// one array G-hat = sqrt|s| G: A fragments are G-hat rows times sign(s), B
// fragments G-hat rows, so sum_q A B = sum_q s G G.
template <int P, int MODE, int R0, int R1>
__device__ __forceinline__ void stiffness_mma(const Out &A, const double *Gm, const double *SGm, int el, double mu,
                                              double lam, int lane) {
  using D = Dims<P>;
  constexpr int NT8 = D::NT8, KS = D::KS, RS = D::RS, NN = D::NN;
  constexpr int NR = R1 - R0;
  double acc[NR][NT8][2];
#pragma unroll
  for (int r = 0; r < NR; r++)
#pragma unroll
    for (int c = 0; c < NT8; c++) acc[r][c][0] = acc[r][c][1] = 0.0;
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int ks = 0; ks < KS; ks++) {
    const int q = 4 * ks + t;
    const double sg = SGm[q];
    double af[NR], bf[NT8];
#pragma unroll
    for (int r = 0; r < NR; r++) af[r] = sg * Gm[q * RS + 8 * (R0 + r) + g];
#pragma unroll
    for (int c = 0; c < NT8; c++)
      if (c >= R0) bf[c] = Gm[q * RS + 8 * c + g];
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
      for (int c = 0; c < NT8; c++)
        if (c >= R0 + r) dmma(acc[r][c][0], acc[r][c][1], af[r], bf[c]);
  }
  const double c11 = lam + 2.0 * mu;
  const int i = g & 1;
#pragma unroll
  for (int r = 0; r < NR; r++) {
    const int a = (8 * (R0 + r) + g) >> 1;
#pragma unroll
    for (int c = 0; c < NT8; c++) {
      if (c < R0 + r) continue;
      const double o0 = __shfl_xor_sync(0xffffffffu, acc[r][c][0], 4);
      const double o1 = __shfl_xor_sync(0xffffffffu, acc[r][c][1], 4);
      const double mxx = i ? o0 : acc[r][c][0], mxy = i ? o1 : acc[r][c][1];
      const double myx = i ? acc[r][c][0] : o0, myy = i ? acc[r][c][1] : o1;
      const int b = 4 * c + t;
      if (a < NN && b < NN && a <= b && (i == 0 || a < b)) {
        const double kxx = c11 * mxx + mu * myy;
        const double kxy = lam * mxy + mu * myx;
        const double kyx = lam * myx + mu * mxy;
        const double kyy = c11 * myy + mu * mxx;
        write_block<P, MODE>(A, el, a, b, i, kxx, kxy, kyx, kyy);
      }
    }
  }
}

// NONLINEAR element stiffness, one warp per node-tile pair (TA <= TB): the four
// component tiles K[(a,i),(b,k)], a in TA, b in TB, share the GA fragment of TA.
// Lane l holds (a, b) = (8TA + l/4, 8TB + 2(l%4) + h) of all four, i.e. whole
// 2x2 blocks; the block (b, a) is written as the transpose (K is symmetric).
template <int P, int MODE>
__device__ __forceinline__ void stiffness_nl(const Out &A, const double *GA, const double *GB, int el, int pair,
                                             int lane) {
  using N = NLDims<P>;
  constexpr int NTN = N::NTN, KSN = N::KSN, RA = N::RA, RB = N::RB, NP = N::NP, NN = N::NN;
  int TA = 0, r = pair;
#pragma unroll
  for (int k = 0; k < NTN; k++)
    if (TA == k && r >= NTN - k) {
      r -= NTN - k;
      TA = k + 1;
    }
  const int TB = TA + r;
  const int g = lane >> 2, t = lane & 3;
  double c[4][2];
#pragma unroll
  for (int j = 0; j < 4; j++) c[j][0] = c[j][1] = 0.0;
  const double *pa = GA + t * RA + 8 * TA + g;
  const double *pb = GB + t * RB + 8 * TB + g;
#pragma unroll 4
  for (int ks = 0; ks < KSN; ks++) {
    const double av = pa[ks * 4 * RA];
    double bv[4];
#pragma unroll
    for (int j = 0; j < 4; j++) bv[j] = pb[ks * 4 * RB + j * NP];
#pragma unroll
    for (int j = 0; j < 4; j++) dmma(c[j][0], c[j][1], av, bv[j]);
  }
  const int a = 8 * TA + g;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int b = 8 * TB + 2 * t + h;
    if (a < NN && b < NN && (TA < TB || a <= b)) {
      write_block<P, MODE>(A, el, a, b, 0, c[0][h], c[1][h], c[2][h], c[3][h]);
      if (a != b) write_block<P, MODE>(A, el, a, b, 1, c[0][h], c[1][h], c[2][h], c[3][h]);
    }
  }
}

template <int P, typename T, int MODE>
constexpr int min_blocks() {
  return ShapeSel<P, MODE>::MINB;
}

// A group's current batch: EPG (or fewer) consecutive elements k0.. of mesh `mesh`
// (always 0 for the single-mesh kernel); ne == 0 ends the loop.
struct Cursor {
  int mesh;
  int ne;
  int64_t k0;
};

// Work source of the single-mesh kernel: batches of [begin, begin+count), strided
// over all groups of the grid.
struct StrideSource {
  static constexpr bool kBatched = false;
  int64_t begin, end, batch, stride;
  int epg;
  __device__ Cursor make(int64_t b) const {
    Cursor c{0, 0, begin + b * epg};
    if (c.k0 < end) c.ne = (int)min((int64_t)epg, end - c.k0);
    return c;
  }
  __device__ Cursor first(int, int) { return make(batch); }
  __device__ void request(const Cursor &, int) {}
  __device__ Cursor next(const Cursor &) {
    batch += stride;
    return make(batch);
  }
};

// A tile of the batched work queue: `count` consecutive (colour-ordered) element
// positions of mesh `mesh`, starting at `begin`.
struct Tile {
  int mesh;
  int count;
  int64_t begin;
};

// Up to kMaxRanges list-position ranges of one mesh assembled by one launch.
constexpr int kMaxRanges = 4;
struct RangeList {
  int n;
  int64_t begin[kMaxRanges], count[kMaxRanges];
};

// Dependency-ordered assembly of one plan in one persistent launch: the list
// positions are cut into groups (the elements of one colour inside one band of
// element ids) and the groups into tiles, listed in dispatch order.  A tile's
// group may write once every group of its dependency list has finished all its
// tiles; the dependencies keep each block's contributions in colour order, so the
// result equals the colour-by-colour launches bit for bit.
struct SchedTile {
  int64_t begin;  // first list position
  int count;      // list positions (even except at the end of a group)
  int group;
  int mesh = 0;   // batches: the mesh's index in the launch's mesh table
};
struct SchedArgs {
  const SchedTile *tiles;
  const int *groupTiles;  // tiles per group
  const int *depPtr;      // CSR over groups: the groups each group waits for
  const int *deps;
  int *status;            // [0] waits that ran out (sticky), [1] tile dispenser, [2 + g] finished tiles of group g
  int ntiles;
  int stallGroup;         // failure injection for tests: no wait ever sees this group finished (-1: none)
  long long waitLimitNs;  // a wait gives up after this long, counts itself in status[0] and lets the tile proceed
};

// Work source of the batched kernel: groups pull tiles from a per-launch queue
// (one atomic counter per launch) and walk their batches.  The argument blocks of
// the meshes the group works on are kept in two shared-memory slots, filled by the
// thread that takes a tile (at most two meshes are live: the current batch's and
// the next one's), so that a batch's gathers do not wait on a global load of its
// mesh's table first.
struct QueueSource {
  static constexpr bool kBatched = true;
  const Tile *tiles;
  int ntiles;
  int *counter;
  int *slot;  // one int in the group's shared memory
  int bar, gt, epg;
  int64_t kend;
  const AsmArgs *meshes;
  AsmArgs *cache;  // [2] in the group's shared memory
  int *cacheMesh;  // [2]: the mesh each slot holds (-1: none)
  // thread 0: the tile after the current one, taken when the current one starts so
  // that the queue atomic's latency -- long behind a later colour's matrix
  // reductions in L2 -- is hidden by the current tile's work
  int ahead = 0;
  __device__ const AsmArgs &args(int m) const { return cacheMesh[0] == m ? cache[0] : cache[1]; }
  // thread 0: the tile's mesh into the slot that the current batch does not use
  __device__ void cache_tile(int t, int curMesh) {
    if (t >= ntiles) return;
    const int m = tiles[t].mesh;
    if (cacheMesh[0] == m || cacheMesh[1] == m) return;
    const int k = cacheMesh[0] == curMesh ? 1 : 0;
    cache[k] = meshes[m];
    cacheMesh[k] = m;
  }
  __device__ Cursor from_tile(int t) {
    Cursor c{0, 0, 0};
    if (t < ntiles) {
      const Tile tl = tiles[t];
      c.mesh = tl.mesh;
      c.k0 = tl.begin;
      kend = tl.begin + tl.count;
      c.ne = (int)min((int64_t)epg, kend - c.k0);
    }
    return c;
  }
  // The second barrier keeps thread 0 from rewriting the slot (request(), when the
  // first batch is also the tile's last) before every thread of the group has read
  // it: a group whose threads took different tiles would mix two meshes' staged
  // block codes and row bases.
  __device__ Cursor first(int tg, int) {
    if (tg == 0) {
      cacheMesh[0] = cacheMesh[1] = -1;
      *slot = atomicAdd(counter, 1);
      ahead = atomicAdd(counter, 1);
      cache_tile(*slot, -1);
    }
    group_sync(bar, gt);
    const Cursor c = from_tile(*slot);
    group_sync(bar, gt);
    return c;
  }
  // Before the group barrier that precedes next(): grab the following tile when
  // this is the tile's last batch.
  __device__ void request(const Cursor &c, int tg) {
    if (tg == 0 && c.k0 + epg >= kend) {
      *slot = ahead;
      cache_tile(ahead, c.mesh);
      if (ahead < ntiles) ahead = atomicAdd(counter, 1);
    }
  }
  __device__ Cursor next(const Cursor &c) {
    if (c.k0 + epg >= kend) return from_tile(*slot);
    Cursor n = c;
    n.k0 = c.k0 + epg;
    n.ne = (int)min((int64_t)epg, kend - n.k0);
    return n;
  }
};

// The per-CTA prologue: derivative table and weights, zeroed MMA padding rows.
template <int P, typename T, int MODE>
__device__ __forceinline__ void cta_prologue(unsigned char *smem) {
  using S = ShapeSel<P, MODE>;
  using L = Layout<P, T, MODE>;
  using D = Dims<P>;
  constexpr int P1 = P + 1, NN = D::NN, NQ = NN, NQP = D::NQP, RS = D::RS, EPG = S::EPG;
  double2 *tabT = reinterpret_cast<double2 *>(smem + L::tabT);
  double *wq = reinterpret_cast<double *>(smem + L::wq);
  for (int i = threadIdx.x; i < NQ * NN; i += blockDim.x) {
    const int q = i / NN, a = i - q * NN;
    double Nx, dNx, Ny, dNy;
    lag1d(P, kGX[P][q % P1], a % P1, Nx, dNx);
    lag1d(P, kGX[P][q / P1], a / P1, Ny, dNy);
    tabT[a * NQ + q] = make_double2(__dmul_rn(Ny, dNx), __dmul_rn(Nx, dNy));
  }
  for (int q = threadIdx.x; q < NQ; q += blockDim.x) wq[q] = __dmul_rn(kGW[P][q % P1], kGW[P][q / P1]);
  __syncthreads();
  // sum_a dN(a, q): zero in exact arithmetic, a few ulp of the table entries in
  // FP64; Neumaier-compensated sum of the table (error ~1e-30 absolute)
  double2 *csum = reinterpret_cast<double2 *>(smem + L::csum);
  for (int q = threadIdx.x; q < NQ; q += blockDim.x) {
    double s0 = 0.0, c0 = 0.0, s1 = 0.0, c1 = 0.0;
    for (int a = 0; a < NN; a++) {
      const double2 d = tabT[a * NQ + q];
      const double t0 = s0 + d.x, t1 = s1 + d.y;
      c0 += fabs(s0) >= fabs(d.x) ? (s0 - t0) + d.x : (d.x - t0) + s0;
      c1 += fabs(s1) >= fabs(d.y) ? (s1 - t1) + d.y : (d.y - t1) + s1;
      s0 = t0;
      s1 = t1;
    }
    csum[q] = make_double2(s0 + c0, s1 + c1);
  }
  if constexpr (L::NL) {
    // padded kappa rows and node columns of GA/GB feed the MMA: zero once (the
    // quadrature stage writes only the real entries)
    constexpr int PER = (int)(L::GH_ELEM / 8);
    for (int i = threadIdx.x; i < S::GPC * EPG * PER; i += blockDim.x) {
      const int g = i / (EPG * PER), r = i - g * EPG * PER;
      unsigned char *gs = smem + L::groups + g * L::group_bytes;
      reinterpret_cast<double *>(gs + L::G)[r] = 0.0;
    }
  } else if constexpr (L::TC) {
    // the padded quadrature rows feed the k dimension of the MMA: zero once
    constexpr int PAD = (NQP - NQ) * RS;
    for (int i = threadIdx.x; i < S::GPC * EPG * PAD; i += blockDim.x) {
      const int g = i / (EPG * PAD), r = i - g * EPG * PAD, el = r / PAD, o = r - el * PAD;
      unsigned char *gs = smem + L::groups + g * L::group_bytes;
      reinterpret_cast<double *>(gs + L::G)[el * NQP * RS + NQ * RS + o] = 0.0;
    }
    for (int i = threadIdx.x; i < S::GPC * EPG * (NQP - NQ); i += blockDim.x) {
      const int g = i / (EPG * (NQP - NQ)), r = i - g * EPG * (NQP - NQ), el = r / (NQP - NQ), o = r - el * (NQP - NQ);
      unsigned char *gs = smem + L::groups + g * L::group_bytes;
      reinterpret_cast<double *>(gs + L::SG)[el * NQP + NQ + o] = 0.0;
    }
  }
  __syncthreads();
}

// One group's assembly loop over the batches its work source yields.  `single`
// is the single-mesh kernel's argument block (read straight from the parameter
// bank); batched sources read `meshes[cursor.mesh]` from global memory.
template <int P, typename T, int MODE, typename Src>
__device__ __forceinline__ void group_loop(unsigned char *smem, Src &src, const AsmArgs &single,
                                           const AsmArgs *__restrict__ meshes) {
  using S = ShapeSel<P, MODE>;
  using L = Layout<P, T, MODE>;
  using D = Dims<P>;
  using ND = NLDims<P>;
  constexpr bool TC = L::TC, NL = L::NL;
  constexpr int P1 = P + 1, NN = D::NN, NQ = NN, NNP = L::NNP, NTILE = D::NTILE;
  constexpr int NQP = D::NQP, RS = D::RS;
  constexpr int GT = S::GT, EPG = S::EPG, NPART = S::NPART, SQ = EPG * NQ;
  static_assert(EPG * NN <= GT, "one prefetched node per thread");
  static_assert(GT % 32 == 0 && 32 % NPART == 0, "group/part shape");
  using T2 = typename Vec2<T>::type;
  const double2 *tabT = reinterpret_cast<const double2 *>(smem + L::tabT);
  const double *wq = reinterpret_cast<const double *>(smem + L::wq);
  const double2 *csum = reinterpret_cast<const double2 *>(smem + L::csum);

  const int g = threadIdx.x / GT, tg = threadIdx.x - g * GT;
  const int warp = tg >> 5, lane = tg & 31;
  unsigned char *gs = smem + L::groups + g * L::group_bytes;
  double2 *X = reinterpret_cast<double2 *>(gs + L::X);
  double2 *U = reinterpret_cast<double2 *>(gs + L::U);
  double *S3 = reinterpret_cast<double *>(gs + L::S3);
  int *nid = reinterpret_cast<int *>(gs + L::nid);
  int *rbase = reinterpret_cast<int *>(gs + L::rbase);
  unsigned char *stage = gs + L::stage;
  constexpr size_t STAGE = align16(L::STAGE);
  const int bar = 1 + g;

  // Gather of the next batch, issued early so its latency overlaps the current batch.
  int pf_node = 0, pf_rb = 0;
  double2 pf_x = make_double2(0, 0), pf_u = make_double2(0, 0);
  auto args = [&](const Cursor &c) -> const AsmArgs & {
    if constexpr (Src::kBatched) {
      return src.args(c.mesh);
    } else {
      return single;
    }
  };
  auto prefetch = [&](const Cursor &c) {
    if (tg >= c.ne * NN) return;
    const AsmArgs &M = args(c);
    const int el = tg / NN, a = tg - el * NN;
    const int64_t k = c.k0 + el;
    if constexpr ((MODE & kPlan) != 0) {
      pf_node = __ldg(M.connList + k * NN + a);
    } else {
      pf_node = __ldg(M.conn + __ldg(M.connPtr + k) + a);
    }
    pf_x = __ldg(reinterpret_cast<const double2 *>(M.coords) + pf_node);
    pf_u = __ldg(reinterpret_cast<const double2 *>(M.states) + pf_node);
    if constexpr ((MODE & (kPlan | kJac)) == (kPlan | kJac) || (MODE & (kPlan | kRes)) == (kPlan | kRes)) {
      pf_rb = __ldg(M.rowp + pf_node);
    }
  };
  // The batch's code records (plan) or element map rows (drop-in Jacobian), copied
  // asynchronously into stage buffer `buf`.
  auto stage_codes = [&](const Cursor &c, int buf) {
    if (c.ne <= 0) return;
    const AsmArgs &M = args(c);
    unsigned char *dst = stage + buf * STAGE;
    if constexpr ((MODE & kPlan) != 0) {
      constexpr int CS = D::CS;
      const unsigned char *src_ = M.blockCode + c.k0 * CS;
      for (int i = tg; i < c.ne * CS / 16; i += GT) cp_async16(dst + 16 * i, src_ + 16 * i);
    } else if constexpr ((MODE & kJac) != 0) {
      const int *src_ = M.map + c.k0 * NN * NN;
      for (int i = tg; i < c.ne * NN * NN; i += GT) cp_async4(dst + 4 * i, src_ + i);
    }
    cp_async_commit();
  };

  // kU: zero the operand tiles once (their padding -- rows 2 NN..63 and K columns
  // NQ..31 -- stays zero), set up the MMA-completion mbarrier, allocate 64 TMEM
  // columns (the 64 x 64 FP32 accumulator)
  uint32_t u_tmem = 0, u_phase = 0;
  if constexpr (L::UM) {
    uint4 *z = reinterpret_cast<uint4 *>(smem + L::uop);
    for (int i = tg; i < 12 * umma::kTileBytes / 16; i += GT) z[i] = make_uint4(0u, 0u, 0u, 0u);
    if (tg == 0) umma::mbar_init(reinterpret_cast<uint64_t *>(smem + L::umbar), 1);
    if (warp == 0) umma::tmem_alloc(reinterpret_cast<uint32_t *>(smem + L::utmem), 64);
    umma::fence_before_sync();
    group_sync(bar, GT);
    umma::fence_after_sync();
    u_tmem = *reinterpret_cast<const uint32_t *>(smem + L::utmem);
  }

  Cursor cur = src.first(tg, bar);
  prefetch(cur);
  stage_codes(cur, 0);
  int buf = 0;
  while (cur.ne > 0) {
    const AsmArgs &M = args(cur);
    const int64_t k0 = cur.k0;
    const int ne = cur.ne;
    const double mu = M.mu, lam = M.lam, thick = M.t;
    const T cMu = T(mu), cLam = T(lam), cC11 = T(lam + 2.0 * mu);
    const Out A{M.mat, M.residual, stage + buf * STAGE, rbase, reinterpret_cast<const int *>(stage + buf * STAGE)};

    // 0. commit the gathered element data
    if (tg < ne * NN) {
      X[tg] = pf_x;
      U[tg] = pf_u;
      nid[tg] = pf_node;
      rbase[tg] = pf_rb;
    }
    cp_async_wait_all();
    src.request(cur, tg);
    group_sync(bar, GT);
    const Cursor nxt = src.next(cur);
    prefetch(nxt);
    stage_codes(nxt, buf ^ 1);

    // 1. quadrature points: NPART lanes per (element, q) split the node sums,
    //    every lane of the quad then forms J^-1 and the gradients of its nodes
    //    (their table entries stay in registers between the two loops).
    //    J = sum_a x_a dN_a cancels by ~h/|x|, so the coordinates enter relative
    //    to the element's node 0 (exact for nearby values) and x_0 sum_a dN_a is
    //    added back: the same sum, evaluated without the cancellation.
    constexpr int MAXJ = (NN + NPART - 1) / NPART;
    for (int base = 0; base < EPG * NQ * NPART; base += GT) {
      const int i = base + tg;
      const int iq = i / NPART, part = i - iq * NPART;
      const int el = iq / NQ, q = iq - el * NQ;
      const bool act = i < EPG * NQ * NPART && el < ne;
      double j00 = 0, j01 = 0, j10 = 0, j11 = 0, g00 = 0, g01 = 0, g10 = 0, g11 = 0;
      const double2 x0 = act ? X[el * NN] : make_double2(0.0, 0.0);
      double2 dt[MAXJ];
#pragma unroll
      for (int j = 0; j < MAXJ; j++) {
        const int a = part + j * NPART;
        dt[j] = make_double2(0.0, 0.0);
        if (act && a < NN) {
          const double2 d = tabT[a * NQ + q];
          dt[j] = d;
          const double2 xa = X[el * NN + a], u = U[el * NN + a];
          const double2 x = make_double2(xa.x - x0.x, xa.y - x0.y);
          j00 = fma(x.x, d.x, j00);
          j01 = fma(x.x, d.y, j01);
          j10 = fma(x.y, d.x, j10);
          j11 = fma(x.y, d.y, j11);
          g00 = fma(u.x, d.x, g00);
          g01 = fma(u.x, d.y, g01);
          g10 = fma(u.y, d.x, g10);
          g11 = fma(u.y, d.y, g11);
        }
      }
#pragma unroll
      for (int o = 1; o < NPART; o <<= 1) {
        j00 += __shfl_xor_sync(0xffffffffu, j00, o);
        j01 += __shfl_xor_sync(0xffffffffu, j01, o);
        j10 += __shfl_xor_sync(0xffffffffu, j10, o);
        j11 += __shfl_xor_sync(0xffffffffu, j11, o);
        g00 += __shfl_xor_sync(0xffffffffu, g00, o);
        g01 += __shfl_xor_sync(0xffffffffu, g01, o);
        g10 += __shfl_xor_sync(0xffffffffu, g10, o);
        g11 += __shfl_xor_sync(0xffffffffu, g11, o);
      }
      if (act) {
        const double2 cs = csum[q];
        j00 = fma(x0.x, cs.x, j00);
        j01 = fma(x0.x, cs.y, j01);
        j10 = fma(x0.y, cs.x, j10);
        j11 = fma(x0.y, cs.y, j11);
        const double det = j00 * j11 - j01 * j10;
        const double inv = 1.0 / det;
        const double i00 = j11 * inv, i01 = -j01 * inv, i10 = -j10 * inv, i11 = j00 * inv;
        const double st = wq[q] * det * thick;
        // FP64: gradients scaled by sqrt|st| (G-hat), the weak stress by st/sqrt|st|
        const double rs = TC ? sqrt(fabs(st)) : 1.0;
        const double sg = st < 0.0 ? -1.0 : 1.0;
        const double sw = TC ? sg * rs : st;
        if constexpr (NL) {
          // F = I + g, Green strain E, S = 2 mu E + lam tr(E) I, first Piola P = F S;
          // tangent A_{il,kn} = delta_ik S_ln + mu F_in F_kl + mu (F F^T)_ik delta_ln + lam F_il F_kn
          const double uxx = g00 * i00 + g01 * i10, uxy = g00 * i01 + g01 * i11;
          const double uyx = g10 * i00 + g11 * i10, uyy = g10 * i01 + g11 * i11;
          const double F[2][2] = {{1.0 + uxx, uxy}, {uyx, 1.0 + uyy}};
          const double e00 = 0.5 * (2.0 * uxx + uxx * uxx + uyx * uyx);
          const double e01 = 0.5 * (uxy + uyx + uxx * uxy + uyx * uyy);
          const double e11 = 0.5 * (2.0 * uyy + uxy * uxy + uyy * uyy);
          const double trE = e00 + e11;
          const double Sm[2][2] = {{2.0 * mu * e00 + lam * trE, 2.0 * mu * e01}, {2.0 * mu * e01, 2.0 * mu * e11 + lam * trE}};
          if (part == 0) {
#pragma unroll
            for (int ii = 0; ii < 2; ii++)
#pragma unroll
              for (int jj = 0; jj < 2; jj++)
                S3[(2 * ii + jj) * SQ + iq] = sw * (F[ii][0] * Sm[0][jj] + F[ii][1] * Sm[1][jj]);
          }
          double Cs[2][2][2][2];  // sign(s) * A_{il,kn}, [i][l][k][n]
#pragma unroll
          for (int ii = 0; ii < 2; ii++)
#pragma unroll
            for (int ll = 0; ll < 2; ll++)
#pragma unroll
              for (int kk = 0; kk < 2; kk++)
#pragma unroll
                for (int nn = 0; nn < 2; nn++) {
                  const double bik = F[ii][0] * F[kk][0] + F[ii][1] * F[kk][1];
                  double v = mu * F[ii][nn] * F[kk][ll] + lam * F[ii][ll] * F[kk][nn];
                  if (ii == kk) v += Sm[ll][nn];
                  if (ll == nn) v += mu * bik;
                  Cs[ii][ll][kk][nn] = sg * v;
                }
          double *GA = reinterpret_cast<double *>(gs + L::G) + el * (L::GH_ELEM / 8);
          double *GB = GA + ND::KN * ND::RA;
#pragma unroll
          for (int j = 0; j < MAXJ; j++) {
            const int a = part + j * NPART;
            if (a >= NN) continue;
            const double2 d = dt[j];
            const double gh[2] = {rs * (d.x * i00 + d.y * i10), rs * (d.x * i01 + d.y * i11)};
#pragma unroll
            for (int ll = 0; ll < 2; ll++) {
              const int kap = ll * NQ + q;
              GA[kap * ND::RA + a] = gh[ll];
#pragma unroll
              for (int ii = 0; ii < 2; ii++)
#pragma unroll
                for (int kk = 0; kk < 2; kk++)
                  GB[kap * ND::RB + (2 * ii + kk) * ND::NP + a] =
                      Cs[ii][ll][kk][0] * gh[0] + Cs[ii][ll][kk][1] * gh[1];
            }
          }
        } else {
        if (part == 0) {
          const double uxx = g00 * i00 + g01 * i10, uxy = g00 * i01 + g01 * i11;
          const double uyx = g10 * i00 + g11 * i10, uyy = g10 * i01 + g11 * i11;
          const double tr = uxx + uyy;
          S3[0 * SQ + iq] = sw * (2.0 * mu * uxx + lam * tr);
          S3[1 * SQ + iq] = sw * (mu * (uxy + uyx));
          S3[2 * SQ + iq] = sw * (2.0 * mu * uyy + lam * tr);
          if constexpr (TC) reinterpret_cast<double *>(gs + L::SG)[el * NQP + q] = sg;
        }
#pragma unroll
        for (int j = 0; j < MAXJ; j++) {
          const int a = part + j * NPART;
          if (a >= NN) continue;
          const double2 d = dt[j];
          const double gx = d.x * i00 + d.y * i10;
          const double gy = d.x * i01 + d.y * i11;
          if constexpr (TC) {
            double *Gm = reinterpret_cast<double *>(gs + L::G) + (el * NQP + q) * RS;
            *reinterpret_cast<double2 *>(Gm + 2 * a) = make_double2(rs * gx, rs * gy);
          } else {
            T2 gv;
            gv.x = T(gx);
            gv.y = T(gy);
            reinterpret_cast<T2 *>(gs + L::G)[iq * NNP + a] = gv;
            if constexpr ((MODE & kJac) != 0) {
              T2 hv;
              hv.x = T(st * gx);
              hv.y = T(st * gy);
              reinterpret_cast<T2 *>(gs + L::H)[iq * NNP + a] = hv;
            }
          }
        }
        }
      }
    }
    group_sync(bar, GT);

    // 2a. residual R_a = sum_q S(q) G_a(q), NPART lanes per node split the q sum (kU: run
    // while the tensor cores form the element stiffness, below)
    auto residual_stage = [&]() {
      for (int base = 0; base < EPG * NN * NPART; base += GT) {
        const int i = base + tg;
        const int ia = i / NPART, part = i - ia * NPART;
        const int el = ia / NN, a = ia - el * NN;
        const bool act = i < EPG * NN * NPART && el < ne;
        T rx = 0, ry = 0;
        if (act) {
#pragma unroll 2
          for (int q = part; q < NQ; q += NPART) {
            const int iq = el * NQ + q;
            T gx, gy;
            if constexpr (NL) {
              const double *GA = reinterpret_cast<const double *>(gs + L::G) + el * (L::GH_ELEM / 8);
              gx = GA[q * ND::RA + a];
              gy = GA[(NQ + q) * ND::RA + a];
              const double pxx = S3[0 * SQ + iq], pxy = S3[1 * SQ + iq];
              const double pyx = S3[2 * SQ + iq], pyy = S3[3 * SQ + iq];
              rx = fma(pxx, gx, fma(pxy, gy, rx));
              ry = fma(pyx, gx, fma(pyy, gy, ry));
              continue;
            } else if constexpr (TC) {
              const double2 gv = *reinterpret_cast<const double2 *>(reinterpret_cast<const double *>(gs + L::G) +
                                                                     (el * NQP + q) * RS + 2 * a);
              gx = gv.x;
              gy = gv.y;
            } else {
              const T2 gv = reinterpret_cast<const T2 *>(gs + L::G)[iq * NNP + a];
              gx = gv.x;
              gy = gv.y;
            }
            const T sxx = T(S3[0 * SQ + iq]), sxy = T(S3[1 * SQ + iq]), syy = T(S3[2 * SQ + iq]);
            rx = fma(sxx, gx, fma(sxy, gy, rx));
            ry = fma(sxy, gx, fma(syy, gy, ry));
          }
        }
#pragma unroll
        for (int o = 1; o < NPART; o <<= 1) {
          rx += __shfl_xor_sync(0xffffffffu, rx, o);
          ry += __shfl_xor_sync(0xffffffffu, ry, o);
        }
        if (act && part == 0) {
          double *dst = A.residual + 2 * (int64_t)nid[ia];
          if constexpr ((MODE & kPlan) != 0) {
            if (A.codes[el * D::CS + NN * NN + a]) {
              *reinterpret_cast<double2 *>(dst) = make_double2(double(rx), double(ry));
            } else {
              atomicAdd(dst, double(rx));
              atomicAdd(dst + 1, double(ry));
            }
          } else {
            atomicAdd(dst, double(rx));
            atomicAdd(dst + 1, double(ry));
          }
        }
      }
    };
    if constexpr ((MODE & kRes) != 0 && !(L::UM && (MODE & kJac) != 0)) residual_stage();

    // 2b. element stiffness
    if constexpr ((MODE & kJac) != 0) {
      if constexpr (NL) {
        // FP64 tensor cores: warps take (element, node-tile pair) work items
        constexpr int NW = GT / 32;
        for (int w = warp; w < ne * ND::NPAIR; w += NW) {
          const int el = w / ND::NPAIR, pair = w - el * ND::NPAIR;
          const double *GA = reinterpret_cast<const double *>(gs + L::G) + el * (L::GH_ELEM / 8);
          stiffness_nl<P, MODE>(A, GA, GA + ND::KN * ND::RA, el, pair, lane);
        }
      } else if constexpr (TC) {
        // FP64 tensor cores: warps take (element, row range) work items
        constexpr int WPE = RowSplit<P>::WPE;  // warps per element
        constexpr int NW = GT / 32;
        for (int w = warp; w < ne * WPE; w += NW) {
          const int el = w / WPE, part = w - el * WPE;
          const double *Gm = reinterpret_cast<const double *>(gs + L::G) + el * NQP * RS;
          const double *Hm = reinterpret_cast<const double *>(gs + L::SG) + el * NQP;
          if constexpr (WPE == 1) {
            stiffness_mma<P, MODE, 0, D::NT8>(A, Gm, Hm, el, mu, lam, lane);
          } else {
            if constexpr (WPE == 2) {
              // p = 3: tile row 0 (4 tiles) | rows 1..3 (3 + 2 + 1 tiles)
              if (part == 0)
                stiffness_mma<P, MODE, 0, 1>(A, Gm, Hm, el, mu, lam, lane);
              else
                stiffness_mma<P, MODE, 1, D::NT8>(A, Gm, Hm, el, mu, lam, lane);
            } else {
              static_assert(P != 4 || D::NT8 == 7, "row split of the 7x7 tile grid");
              if (part == 0)
                stiffness_mma<P, MODE, 0, 1>(A, Gm, Hm, el, mu, lam, lane);
              else if (part == 1)
                stiffness_mma<P, MODE, 1, 2>(A, Gm, Hm, el, mu, lam, lane);
              else if (part == 2)
                stiffness_mma<P, MODE, 2, 4>(A, Gm, Hm, el, mu, lam, lane);
              else
                stiffness_mma<P, MODE, 4, D::NT8>(A, Gm, Hm, el, mu, lam, lane);
            }
          }
        }
      } else if constexpr (L::UM) {
        // tcgen05: M[(a,i),(b,j)] = sum_q H_i(q,a) G_j(q,b) as one 64 x 64 x 32 product per
        // element (rows r = 2a + i and columns n = 2b + j padded from 50 to 64, K = the 25
        // quadrature points padded to 32), each FP32 operand split into three BF16 parts
        // and the six part products (lo.hi, hi.lo, mid.mid, mid.hi, hi.mid, hi.hi;
        // ~FP32 accuracy, as the fragment kernel's order-3 form) accumulated in FP32 in
        // TMEM: 12 MMAs of 64 x 64 x 16 issued by one thread.
        unsigned char *uop = smem + L::uop;
        uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + L::umbar);
        const T2 *G = reinterpret_cast<const T2 *>(gs + L::G);
        const T2 *H = reinterpret_cast<const T2 *>(gs + L::H);
        // operands: (A = H | B = G, chunk of 8 quadrature points, row r < 2 NN), rows
        // fastest: a quarter-warp stores eight consecutive rows' 16-byte K runs, eight
        // distinct bank groups of one tile
        constexpr int NR = 2 * NN, NCH = 4;
        for (int it = tg; it < 2 * NR * NCH; it += GT) {
          const int op = it / (NR * NCH), rem = it - op * NR * NCH;
          const int c = rem / NR, r = rem - c * NR;
          const int a = r >> 1, i = r & 1;
          const T2 *src_ = op ? G : H;
          uint32_t w[3][4];
#pragma unroll
          for (int j = 0; j < 8; j += 2) {
            float v2[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const int q = 8 * c + j + h;
              const T2 gv = q < NQ ? src_[q * NNP + a] : T2{0.0f, 0.0f};
              v2[h] = i ? gv.y : gv.x;
            }
            uint32_t pk[3] = {0u, 0u, 0u};
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const __nv_bfloat16 hi = __float2bfloat16_rn(v2[h]);
              const float r1 = v2[h] - __bfloat162float(hi);
              const __nv_bfloat16 mid = __float2bfloat16_rn(r1);
              const __nv_bfloat16 lo = __float2bfloat16_rn(r1 - __bfloat162float(mid));
              pk[0] |= (uint32_t)__bfloat16_as_ushort(hi) << (16 * h);
              pk[1] |= (uint32_t)__bfloat16_as_ushort(mid) << (16 * h);
              pk[2] |= (uint32_t)__bfloat16_as_ushort(lo) << (16 * h);
            }
#pragma unroll
            for (int pt = 0; pt < 3; pt++) w[pt][j >> 1] = pk[pt];
          }
#pragma unroll
          for (int pt = 0; pt < 3; pt++) {
            unsigned char *tile = uop + ((op * 3 + pt) * 2 + (c >> 1)) * umma::kTileBytes;
            *reinterpret_cast<uint4 *>(tile + umma::tile_offset(r, 8 * (c & 1))) =
                make_uint4(w[pt][0], w[pt][1], w[pt][2], w[pt][3]);
          }
        }
        umma::fence_smem_to_async();
        umma::fence_before_sync();
        group_sync(bar, GT);
        umma::fence_after_sync();
        if (tg == 0) {
          // smallest part products first: (A part, B part) = (lo, hi), (hi, lo), (mid, mid), (mid, hi), (hi, mid), (hi, hi)
          constexpr int pa[6] = {2, 0, 1, 1, 0, 0}, pb[6] = {0, 2, 1, 0, 1, 0};
          const uint32_t base = umma::smem_u32(uop);
#pragma unroll
          for (int k = 0; k < 6; k++)
#pragma unroll
            for (int ks = 0; ks < 2; ks++)
              umma::mma_bf16(u_tmem, umma::smem_desc(base + ((0 * 3 + pa[k]) * 2 + ks) * umma::kTileBytes),
                             umma::smem_desc(base + ((1 * 3 + pb[k]) * 2 + ks) * umma::kTileBytes),
                             umma::kIdescBF16_M64N64, (k | ks) != 0);
          umma::commit(mbar);
        }
        if constexpr ((MODE & kRes) != 0) residual_stage();
        // one thread waits for the MMAs (bounded), the group follows through its barrier
        if (tg == 0 && !umma::mbar_wait(mbar, u_phase, 1u << 20) && M.waits) atomicAdd(M.waits, 1);
        u_phase ^= 1u;
        umma::fence_before_sync();
        group_sync(bar, GT);
        umma::fence_after_sync();
        // epilogue: lanes 0-15 of warp w hold accumulator rows 16 w + lane; they stage
        // the 2 NN valid rows in shared memory (over the operand tiles, free now), then
        // all threads combine and write the upper-triangle blocks and their transposes
        // The staging covers only A tiles (the first 6 x 2 KB): the next element rewrites
        // their rows 0 .. 2 NN - 1 over all 32 K columns (zeros past NQ), and what stays in
        // rows 2 NN .. 63 reaches only accumulator rows nobody reads; the B tiles keep
        // their zero padding.
        // staged row stride in floats: an odd number of float2 pairs, so that the 16 rows a
        // warp stores land on 16 distinct bank pairs
        constexpr int AS = (NN % 2) ? 2 * NN : 2 * NN + 2;
        static_assert(NR * AS * 4 <= 6 * umma::kTileBytes, "staged accumulator fits the A operand tiles");
        float *acc = reinterpret_cast<float *>(uop);
        {
          const int r = 16 * warp + (lane & 15);
#pragma unroll 1
          for (int cc = 0; cc < (NR + 15) / 16; cc++) {
            float v[16];
            umma::tmem_ld16(u_tmem + ((uint32_t)(32 * warp) << 16) + 16 * cc, v);
            if (lane < 16 && r < NR) {
#pragma unroll
              for (int j = 0; j < 16; j += 2)
                if (16 * cc + j < NR)
                  *reinterpret_cast<float2 *>(acc + r * AS + 16 * cc + j) = make_float2(v[j], v[j + 1]);
            }
          }
        }
        umma::fence_before_sync();
        group_sync(bar, GT);
        constexpr int NUP = NN * (NN + 1) / 2;
        for (int u = tg; u < NUP; u += GT) {
          // u -> (a, b), a <= b, row-major over the upper triangle
          int a = 0, rem = u;
          while (rem >= NN - a) {
            rem -= NN - a;
            a++;
          }
          const int b = a + rem;
          const float2 m0 = *reinterpret_cast<const float2 *>(acc + (2 * a) * AS + 2 * b);
          const float2 m1 = *reinterpret_cast<const float2 *>(acc + (2 * a + 1) * AS + 2 * b);
          const double mxx = m0.x, mxy = m0.y, myx = m1.x, myy = m1.y;
          const double kxx = (lam + 2.0 * mu) * mxx + mu * myy, kxy = lam * mxy + mu * myx;
          const double kyx = lam * myx + mu * mxy, kyy = (lam + 2.0 * mu) * myy + mu * mxx;
          write_block<P, MODE>(A, 0, a, b, 0, kxx, kxy, kyx, kyy);
          if (a != b) write_block<P, MODE>(A, 0, a, b, 1, kxx, kxy, kyx, kyy);
        }
      } else {
        // FP32 CUDA cores: one (p+1)-row tile x one column per thread, upper triangle
        const T2 *G = reinterpret_cast<const T2 *>(gs + L::G);
        const T2 *H = reinterpret_cast<const T2 *>(gs + L::H);
        for (int i = tg; i < ne * NTILE; i += GT) {
          const int el = i / NTILE;
          int r = i - el * NTILE, at = 0;
#pragma unroll
          for (int row = 0; row < P1; row++) {
            const int len = NN - row * P1;
            if (at == row && r >= len) {
              r -= len;
              at = row + 1;
            }
          }
          const int b = at * P1 + r;
          T m[P1][4];
#pragma unroll
          for (int ax = 0; ax < P1; ax++) m[ax][0] = m[ax][1] = m[ax][2] = m[ax][3] = T(0);
          const T2 *Gb = G + el * NQ * NNP + b;
          const T2 *Ha = H + el * NQ * NNP + at * P1;
#pragma unroll 2
          for (int q = 0; q < NQ; q++) {
            const T2 gv = Gb[q * NNP];
#pragma unroll
            for (int ax = 0; ax < P1; ax++) {
              const T2 hv = Ha[q * NNP + ax];
              m[ax][0] = fma(hv.x, gv.x, m[ax][0]);
              m[ax][1] = fma(hv.x, gv.y, m[ax][1]);
              m[ax][2] = fma(hv.y, gv.x, m[ax][2]);
              m[ax][3] = fma(hv.y, gv.y, m[ax][3]);
            }
          }
#pragma unroll
          for (int ax = 0; ax < P1; ax++) {
            const int a = at * P1 + ax;
            if (a > b) continue;
            const double kxx = double(cC11 * m[ax][0] + cMu * m[ax][3]);
            const double kxy = double(cLam * m[ax][1] + cMu * m[ax][2]);
            const double kyx = double(cLam * m[ax][2] + cMu * m[ax][1]);
            const double kyy = double(cC11 * m[ax][3] + cMu * m[ax][0]);
            write_block<P, MODE>(A, el, a, b, 0, kxx, kxy, kyx, kyy);
            if (a != b) write_block<P, MODE>(A, el, a, b, 1, kxx, kxy, kyx, kyy);
          }
        }
      }
    }
    group_sync(bar, GT);
    cur = nxt;
    buf ^= 1;
  }
  cp_async_wait_all();
  if constexpr (L::UM) {
    umma::fence_before_sync();
    group_sync(bar, GT);
    if (warp == 0) umma::tmem_dealloc(u_tmem, 64);
  }
}

// Single mesh: A.count elements from A.begin, persistent grid-stride over batches.
template <int P, typename T, int MODE>
__global__ void __launch_bounds__(ShapeSel<P, MODE>::GT *ShapeSel<P, MODE>::GPC, min_blocks<P, T, MODE>())
    assemble_kernel(const __grid_constant__ AsmArgs A) {
  using S = ShapeSel<P, MODE>;
  extern __shared__ __align__(16) unsigned char smem[];
  cta_prologue<P, T, MODE>(smem);
  const int g = threadIdx.x / S::GT;
  StrideSource src{A.begin, A.begin + A.count, (int64_t)blockIdx.x * S::GPC + g, (int64_t)gridDim.x * S::GPC,
                   S::EPG};
  group_loop<P, T, MODE>(smem, src, A, nullptr);
}

// Many meshes of one order: groups pull tiles from the launch's queue.
template <int P, typename T, int MODE>
__global__ void __launch_bounds__(ShapeSel<P, MODE>::GT *ShapeSel<P, MODE>::GPC, min_blocks<P, T, MODE>())
    assemble_batched_kernel(const AsmArgs *__restrict__ meshes, const Tile *__restrict__ tiles, int ntiles,
                            int *counter) {
  using S = ShapeSel<P, MODE>;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int slots[S::GPC];
  __shared__ AsmArgs argCache[S::GPC][2];
  __shared__ int argMesh[S::GPC][2];
  cta_prologue<P, T, MODE>(smem);
  const int g = threadIdx.x / S::GT;
  QueueSource src{tiles, ntiles, counter, &slots[g], 1 + g, S::GT, S::EPG, 0, meshes, argCache[g], argMesh[g]};
  group_loop<P, T, MODE>(smem, src, meshes[0], meshes);
}

}  // namespace dev
}  // namespace fem
