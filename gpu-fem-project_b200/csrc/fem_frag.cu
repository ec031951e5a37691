// Warp-fragment assembly kernel: FP64 residual + Jacobian assembly, LINEAR strain at
// orders 2 to 4 and NONLINEAR (Green) strain at orders 2 and 3; FEM_PRECISION_MIXED at
// order 3 with the element stiffness as BF16x6 tensor-core products (which paths use
// it: frag_supported and b16_stiffness at the end of this file).  Launch forms: one
// list-position range (plans, drop-in), up to four ranges (the band-split launches of
// fem_plan_assemble_host), tile queues (batches, the server).
//
// The element kernel in fem_device.cuh stages every element's coordinates,
// states and scaled gradients in shared memory and reads them back for each
// stage; at p = 3 that is ~400 shared-memory wavefronts per element and the
// L1 data pipe, not HBM, bounds it.  Here a warp assembles two elements per
// step and keeps their data in registers laid out as FP64 tensor-core
// (mma.m8n8k4) fragments:
//
//   1. gather    lane (g, t) (g = lane/4, t = lane%4) loads component c = g%4
//                (x, y, u, v) of node 4ks + t of element g/4: that register IS
//                the A fragment of step 2 (rows = 2 elements x 4 components,
//                k = element nodes).  Node ids are read two steps ahead, the
//                coordinates/states one step ahead.
//   2. J stage   C[(e,c)][(q,d)] = sum_a X[(e,c)][a] dN_d(a, q): the isoparametric
//                Jacobian and the reference-space state gradient of both
//                elements at every quadrature point (K4 x K4 MMAs), with the
//                derivative table as B fragments (shared memory, lane order).
//   3. transpose three xor-shuffle rounds per group of four column tiles give each
//                lane all eight values of one quadrature point q = 4(4m + c) + t
//                (one point per lane at p <= 3, two at p = 4); it forms det J, J^-1,
//                s = w det J t, the weak stress and sqrt|s| J^-1 (FP64) and
//                stores the ~10 doubles of q to shared memory.
//   4. fragments lane (g, t) builds G-hat_i(q, a) = sqrt|s| (dN(a,q) J^-1)_i for
//                q = 4ks + t from sqrt|s| J^-1 and the table: the A and B fragments
//                of M_ij[a][b] = sum_q s G_ai G_bj.
//   5. residual  R_(a,i) = sum_q sum_j G-hat_j S-hat_ij on the FP64 pipe from the
//                same fragments, reduced over the lanes of a node by shuffles.
//   6. stiffness p = 2, 3: component-major node tiles (a = 8T + pi(g), pi(g) =
//                4(g%2) + g/2; pairs TA <= TB, four (i, j) tiles sharing
//                fragments, k-steps outermost): lane (g, t) ends with WHOLE 2x2
//                blocks (a, b = 8TB + 4h + t), so the plane-stress combination
//                needs no shuffle and a warp store covers eight runs of four
//                consecutive blocks.  p = 4: interleaved rows r = 2a + i in seven
//                tiles (a = 4T + g/2), one pass per group of tile pairs with the
//                group's fragments rebuilt from the table (the residual rides on
//                the first three groups); lanes l, l^4 exchange the two rows of a
//                block.  Blocks above the diagonal are also written transposed.
//
// Writes.  Plan mode: a launch is one colour; the first contributor of a block
// stores it (one 256-bit store); a later colour adds its 2x2 blocks with
// asynchronous bulk reductions (cp.reduce.async.bulk .add.f64 from shared memory)
// instead of four FP64 L2 atomics per block -- at p = 3 staged by row run, one
// 128-byte reduction per run of four adjacent blocks.  Drop-in mode (reference
// element map, accumulate-into) adds every block that way.  Residual rows: first
// writer stores, others add with atomics.  The arithmetic is the closed form of
// the reference's per-column forward AD (element/FEKernels.h:286-315, 884-976)
// that the element kernel documents.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <type_traits>

#include "fem_common.h"
#include "fem_device.cuh"
#include "fem_launch.h"

// Resident CTAs per SM the register budget is sized for: 3 (168 registers) at
// p = 3, where the 12 live stiffness accumulators need them, and at p = 4; 4 (128)
// at p = 2 and for the residual alone (no stiffness accumulators).
#ifndef FEM_FRAG_MINB
#define FEM_FRAG_MINB ((P == 2 || (MODE & kJac) == 0) ? 4 : 3)
#endif

namespace fem {
namespace dev {

template <int P>
struct FragDims {
  static constexpr int P1 = P + 1, NN = P1 * P1, NQ = NN;
  static constexpr int K4 = (NN + 3) / 4;   // node k-steps = quadrature k-steps = J column tiles
  static constexpr int NQP = 4 * K4;        // padded quadrature points
  static constexpr int NTN = (NN + 7) / 8;  // node tiles of the component-major stiffness product
  static constexpr int CS = Dims<P>::CS;    // plan code record bytes per element
  static constexpr int WARPS = 4;           // warps per CTA
  static constexpr int TG = (K4 + 3) / 4;   // transpose groups: quadrature points per lane
  // Stiffness layout: component-major node tiles at p = 2, 3 (two tiles of 8 nodes),
  // interleaved rows r = 2a + i at p = 4 (50 rows in seven tiles, where node tiles
  // would pad 25 nodes to 32 and need 280 instead of 196 MMAs per element).
  static constexpr bool IL = (P == 4);
  static constexpr int NTAB = IL ? K4 : NTN;  // table tiles per k-step
  static constexpr int TABW = IL ? 16 : 32;   // table entries per (k-step, tile): lane, or (g/2, t)
  static_assert(P >= 2 && P <= 4 && (IL || NTN == 2), "fragment kernel: orders 2 to 4");
};

template <int V>
using IC = std::integral_constant<int, V>;

// Shared memory: CTA tables, then one region per warp.  DROP: drop-in mode (the
// stage holds the reference element map rows, NN*NN ints per element, instead of
// plan code records).  B16: the BF16x6 stiffness table follows the CTA tables.
// JAC = false (residual only): no block staging slots.
template <int P, bool DROP = false, bool NL = false, bool B16 = false, bool JAC = true>
struct FragLayout {
  using F = FragDims<P>;
  static constexpr int K4 = F::K4, NTN = F::NTN, NQP = F::NQP, NN = F::NN;
  static constexpr int CS = DROP ? 4 * NN * NN : F::CS;  // staged bytes per element
  static constexpr size_t tabJ = 0;                          // double [K4][K4][32]
  static constexpr size_t tabF = tabJ + 8 * K4 * K4 * 32;    // double2 [K4][NTAB][TABW]
  static constexpr size_t wq = tabF + 16 * K4 * F::NTAB * F::TABW;  // double [NQP]
  static constexpr size_t csum = align16(wq + 8 * NQP);       // double2 [NQP]: sum_a dN(a, q)
  static constexpr size_t tabB = align16(csum + 16 * NQP);    // double2 [8][32]: BF16x6 stiffness operands
  static constexpr size_t warps = align16(tabB + (B16 ? 16 * 8 * 32 : 0));
  // warp-relative; [2] = the two elements of the step
  static constexpr size_t WI0 = 0;                 // double2 [2][NQP]: sqrt|s| (J^-1_0x, J^-1_1x)
  static constexpr size_t WI1 = WI0 + 16 * 2 * NQP;  // double2 [2][NQP]: sqrt|s| (J^-1_0y, J^-1_1y)
  static constexpr size_t WS0 = WI1 + 16 * 2 * NQP;  // double2 [2][NQP]: (S-hat_xx, S-hat_xy)
  static constexpr size_t WS1 = WS0 + 16 * 2 * NQP;  // double2 [2][NQP]: (S-hat_xy, S-hat_yy)
  static constexpr size_t SG = WS1 + 16 * 2 * NQP;   // double [2][NQP]: sign of s (0 on padding)
  static constexpr size_t NID = SG + 8 * 2 * NQP;    // int [2][NN]: node ids
  static constexpr size_t RB = align16(NID + 4 * 2 * NN);  // int [2][NN]: rowp[node]
  static constexpr size_t STAGE = align16(RB + 4 * 2 * NN);  // [2 buffers][2 elements][CS] code records
  // staging slots: p = 3, 3 node-tile pairs x 2 halves, direct and transposed; p = 2,
  // the (at most 8) blocks one lane writes per element; p = 4, a ring of 4 per lane
  static constexpr int NSLOT = F::IL ? 4 : 8;
  static constexpr size_t REDS = align16(STAGE + 2 * 2 * CS);  // double4 [NSLOT][32]: bulk-reduction sources
  // NONLINEAR: sign(s) x tangent modulus, double [2][NQP][2 (l)][8 (i, k, n)]
  static constexpr size_t AT = align16(REDS + (JAC ? 32 * NSLOT * 32 : 0));
  static constexpr size_t warp_bytes = align16(AT + (NL ? 8 * 2 * NQP * 16 : 0));
  static constexpr size_t total = warps + F::WARPS * warp_bytes;
};

// D += A B, m16n8k16, BF16 operands, FP32 accumulate.
__device__ __forceinline__ void bmma(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
               : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// v ~ hi + mid + lo, three BF16 parts (8 significant bits each, 24 together): the
// FP32 value and its two successive remainders, each rounded to nearest.
__device__ __forceinline__ void split3(double v, uint32_t &hi, uint32_t &mid, uint32_t &lo) {
  const float f = __double2float_rn(v);
  const __nv_bfloat16 h = __float2bfloat16_rn(f);
  const float r1 = f - __bfloat162float(h);
  const __nv_bfloat16 m = __float2bfloat16_rn(r1);
  const __nv_bfloat16 l = __float2bfloat16_rn(r1 - __bfloat162float(m));
  hi = __bfloat16_as_ushort(h);
  mid = __bfloat16_as_ushort(m);
  lo = __bfloat16_as_ushort(l);
}

__device__ __forceinline__ double sel4(double x0, double x1, double x2, double x3, int i) {
  return i == 0 ? x0 : (i == 1 ? x1 : (i == 2 ? x2 : x3));
}

template <int P, bool B16 = false>
__device__ __forceinline__ void frag_prologue(unsigned char *smem) {
  using F = FragDims<P>;
  using L = FragLayout<P, false, false, B16>;
  constexpr int P1 = F::P1, NN = F::NN, NQ = F::NQ, K4 = F::K4, NTAB = F::NTAB, TABW = F::TABW;
  double *tabJ = reinterpret_cast<double *>(smem + L::tabJ);
  double2 *tabF = reinterpret_cast<double2 *>(smem + L::tabF);
  double *wq = reinterpret_cast<double *>(smem + L::wq);
  // dN(a, q) = (N_y dN_x, N_x dN_y) with the rounding of the element kernel's table
  auto dN = [&](int a, int q) {
    double Nx, dNx, Ny, dNy;
    lag1d(P, kGX[P][q % P1], a % P1, Nx, dNx);
    lag1d(P, kGX[P][q / P1], a / P1, Ny, dNy);
    return make_double2(__dmul_rn(Ny, dNx), __dmul_rn(Nx, dNy));
  };
  // J-stage B fragments: lane (g, t) of (ks, tn) holds dN_{g%2}(a = 4ks + t, q = 4tn + g/2)
  for (int i = threadIdx.x; i < K4 * K4 * 32; i += blockDim.x) {
    const int lane = i & 31, blk = i >> 5, ks = blk / K4, tn = blk - ks * K4;
    const int g = lane >> 2, t = lane & 3;
    const int a = 4 * ks + t, q = 4 * tn + (g >> 1);
    double v = 0.0;
    if (a < NN && q < NQ) {
      const double2 d = dN(a, q);
      v = (g & 1) ? d.y : d.x;
    }
    tabJ[i] = v;
  }
  // stiffness fragments at (ks, T), q = 4ks + t: component-major, lane (g, t) holds
  // dN(a = 8T + pi(g), q); interleaved, entry 4(g/2) + t holds dN(a = 4T + g/2, q)
  for (int i = threadIdx.x; i < K4 * NTAB * TABW; i += blockDim.x) {
    const int e = i % TABW, blk = i / TABW, ks = blk / NTAB, T = blk - ks * NTAB;
    int a, q;
    if constexpr (F::IL) {
      a = 4 * T + (e >> 2);
      q = 4 * ks + (e & 3);
    } else {
      const int g = e >> 2, t = e & 3;
      a = 8 * T + 4 * (g & 1) + (g >> 1);
      q = 4 * ks + t;
    }
    tabF[i] = (a < NN && q < NQ) ? dN(a, q) : make_double2(0.0, 0.0);
  }
  for (int q = threadIdx.x; q < F::NQP; q += blockDim.x)
    wq[q] = q < NQ ? __dmul_rn(kGW[P][q % P1], kGW[P][q / P1]) : 0.0;
  // BF16x6 stiffness (order 3): entry (2k + h, lane (g, t)) holds dN(a, q) for the
  // node a = 8h + pi(g) and quadrature point q = 2t + (k & 1) + 8 (k >> 1) that lane
  // (g, t) places in its m16n8k16 fragments
  if constexpr (B16) {
    double2 *tabB = reinterpret_cast<double2 *>(smem + L::tabB);
    for (int i = threadIdx.x; i < 8 * 32; i += blockDim.x) {
      const int lane = i & 31, k = (i >> 5) >> 1, h = (i >> 5) & 1, g = lane >> 2, t = lane & 3;
      const int a = 8 * h + 4 * (g & 1) + (g >> 1), q = 2 * t + (k & 1) + 8 * (k >> 1);
      tabB[i] = (a < NN && q < NQ) ? dN(a, q) : make_double2(0.0, 0.0);
    }
  }
  // sum_a dN(a, q): zero in exact arithmetic, a few ulp of the table entries in
  // FP64; summed with Neumaier compensation (error ~1e-30 absolute) over the J-stage
  // table entries written above (lane (g, t) of block (ks, tn) holds component g%2 of
  // dN(4ks + t, 4tn + g/2)) instead of evaluating the basis again
  __syncthreads();
  double2 *csum = reinterpret_cast<double2 *>(smem + L::csum);
  for (int q = threadIdx.x; q < F::NQP; q += blockDim.x) {
    double s0 = 0.0, c0 = 0.0, s1 = 0.0, c1 = 0.0;
    if (q < NQ) {
      for (int a = 0; a < NN; a++) {
        const int e = (((a >> 2) * K4 + (q >> 2)) * 32) + ((2 * (q & 3)) << 2) + (a & 3);
        const double2 d = make_double2(tabJ[e], tabJ[e + 4]);
        const double t0 = s0 + d.x, t1 = s1 + d.y;
        c0 += fabs(s0) >= fabs(d.x) ? (s0 - t0) + d.x : (d.x - t0) + s0;
        c1 += fabs(s1) >= fabs(d.y) ? (s1 - t1) + d.y : (d.y - t1) + s1;
        s0 = t0;
        s1 = t1;
      }
    }
    csum[q] = make_double2(s0 + c0, s1 + c1);
  }
  __syncthreads();
}

// Staging slot of node-tile pair k (0: (0,0), 1: (0,1), 2: (1,1)), half h, and
// direct (0) / transposed (1) blocks.
__host__ __device__ constexpr int frag_slot(int k, int h, int w) { return k == 0 ? h : (k == 1 ? 2 + 2 * h + w : 6 + h); }

// The block (a, b) of element el (or its transpose (b, a) with w = 1): plan mode
// stores it when this element is its first contributor; otherwise (and in
// drop-in mode always) it goes to its staging position for frag_issue_run.
template <int P, bool PLAN>
__device__ __forceinline__ void frag_put(const Out &O, int el, int a, int b, int w, double kxx, double kxy,
                                         double kyx, double kyy, double *stg) {
  constexpr int NN = Dims<P>::NN, CS = Dims<P>::CS;
  const int r0 = w ? b : a, c0 = w ? a : b;
  const double v0 = kxx, v1 = w ? kyx : kxy, v2 = w ? kxy : kyx, v3 = kyy;
  if constexpr (PLAN) {
    const uint8_t code = O.codes[el * CS + r0 * NN + c0];
    if (code & 0x80) {
      store_block(O.mat + 4 * ((int64_t)O.rbase[el * NN + r0] + (code & 0x7f)), v0, v1, v2, v3);
      return;
    }
  }
  reinterpret_cast<double2 *>(stg)[0] = make_double2(v0, v1);
  reinterpret_cast<double2 *>(stg)[1] = make_double2(v2, v3);
}

// Before the second element of a step writes.  In a plan's pair layout it shares an
// edge with the first: where the first stored a shared block (a generic-proxy
// 256-bit store) the second adds to it with a bulk reduction (async proxy, maybe
// another lane), and where both add (an earlier colour stored it) the first one's
// reduction must land first, or the two would round in either order.  So: wait
// for this lane's reductions to complete, order the lanes, order the proxies.
// Residual rows go generic store or atomic, then atomics: the barrier orders them.
// The order-3 writers, which store first and reduce last, take the two halves
// apart (pair_first_landed before, pair_first_visible after the barrier that
// precedes their reductions) so that the first element's reductions have the second
// element's stores to land in.
__device__ __forceinline__ void pair_first_landed() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void pair_first_visible() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ void pair_order_fence() {
  pair_first_landed();
  __syncwarp();
  pair_first_visible();
}

__device__ __forceinline__ void bulk_add(double *gdst, const double *src, int bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(src);
  asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], %2;" ::"l"(gdst), "r"(sa),
               "r"(bytes)
               : "memory");
}

// Run r of staging slot sl (see frag_slot): four blocks of one matrix row with four
// consecutive element-local columns.  Blocks to add: drop-in, every valid block;
// plan, the valid blocks whose code is not a first store.  One 128-byte reduction
// when all four are added and adjacent in the matrix, else 32 bytes per block
// (four FP64 atomics for a block whose address is not 16-byte aligned).
template <int P, bool PLAN>
__device__ __forceinline__ void frag_issue_run(const Out &O, int el, int sl, int r, const double *redsW) {
  constexpr int NN = Dims<P>::NN, CS = Dims<P>::CS;
  const int k = sl < 2 ? 0 : (sl < 6 ? 1 : 2);
  const int h = sl < 2 ? sl : (sl < 6 ? (sl - 2) >> 1 : sl - 6);
  const int w = (sl >= 2 && sl < 6) ? ((sl - 2) & 1) : 0;
  const int TA = k == 2 ? 1 : 0, TB = k == 0 ? 0 : 1;
  int row, col0, pos0;
  if (w == 0) {
    row = 8 * TA + 4 * (r & 1) + (r >> 1);  // pi(r)
    col0 = 8 * TB + 4 * h;
    pos0 = 4 * r;
  } else {
    const int tt = r >> 1, half = r & 1;
    row = 8 * TB + 4 * h + tt;
    col0 = 8 * TA + 4 * half;
    pos0 = 8 * tt + 4 * half;
  }
  if (row >= NN) return;
  double *dst[4];
  bool add[4];
  bool all = true, adj = true;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int col = col0 + j;
    add[j] = col < NN;
    dst[j] = O.mat;
    if (add[j]) {
      if constexpr (PLAN) {
        const uint8_t code = O.codes[el * CS + row * NN + col];
        add[j] = !(code & 0x80);
        dst[j] = O.mat + 4 * ((int64_t)O.rbase[el * NN + row] + (code & 0x7f));
      } else {
        dst[j] = O.mat + O.map[(el * NN + row) * NN + col];
      }
    }
    all = all && add[j];
    if (j > 0) adj = adj && dst[j] == dst[0] + 4 * j;
  }
  const double *src = redsW + 128 * sl + 4 * pos0;
  if (all && adj && (reinterpret_cast<uintptr_t>(dst[0]) & 15u) == 0) {
    bulk_add(dst[0], src, 128);
    return;
  }
#pragma unroll
  for (int j = 0; j < 4; j++) {
    if (!add[j]) continue;
    if ((reinterpret_cast<uintptr_t>(dst[j]) & 15u) == 0) {
      bulk_add(dst[j], src + 4 * j, 32);
    } else {
      atomicAdd(dst[j] + 0, src[4 * j + 0]);
      atomicAdd(dst[j] + 1, src[4 * j + 1]);
      atomicAdd(dst[j] + 2, src[4 * j + 2]);
      atomicAdd(dst[j] + 3, src[4 * j + 3]);
    }
  }
}

// Per-block writers (order 2, where four consecutive element-local nodes straddle
// grid rows and row runs never merge).  One 2x2 block of element `el` (staged codes /
// row bases in O): a 256-bit store
// when this element is the block's first contributor, else a 32-byte bulk
// reduction from `slot` (this lane's staging slot; the caller has waited for the
// slot's previous bulk read).  `which` = 1 writes the transposed block (b, a).
template <int P>
__device__ __forceinline__ void frag_write(const Out &O, int el, int a, int b, int which, double kxx, double kxy,
                                           double kyx, double kyy, double *slot) {
  constexpr int NN = Dims<P>::NN, CS = Dims<P>::CS;
  const int r0 = which ? b : a, c0 = which ? a : b;
  const double v0 = kxx, v1 = which ? kyx : kxy, v2 = which ? kxy : kyx, v3 = kyy;
  const uint8_t code = O.codes[el * CS + r0 * NN + c0];
  double *blk = O.mat + 4 * ((int64_t)O.rbase[el * NN + r0] + (code & 0x7f));
  if (code & 0x80) {
    store_block(blk, v0, v1, v2, v3);
  } else {
    reinterpret_cast<double2 *>(slot)[0] = make_double2(v0, v1);
    reinterpret_cast<double2 *>(slot)[1] = make_double2(v2, v3);
    const unsigned sa = (unsigned)__cvta_generic_to_shared(slot);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], 32;" ::"l"(blk), "r"(sa)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  }
}

// frag_write without its fence and bulk reduction: a first store goes out at once
// (returns nullptr); a block to add is staged in `slot` and its destination
// returned, for the caller to issue after one proxy fence for all its slots.
template <int P>
__device__ __forceinline__ double *frag_stage(const Out &O, int el, int a, int b, int which, double kxx, double kxy,
                                              double kyx, double kyy, double *slot) {
  constexpr int NN = Dims<P>::NN, CS = Dims<P>::CS;
  const int r0 = which ? b : a, c0 = which ? a : b;
  const double v0 = kxx, v1 = which ? kyx : kxy, v2 = which ? kxy : kyx, v3 = kyy;
  const uint8_t code = O.codes[el * CS + r0 * NN + c0];
  double *blk = O.mat + 4 * ((int64_t)O.rbase[el * NN + r0] + (code & 0x7f));
  if (code & 0x80) {
    store_block(blk, v0, v1, v2, v3);
    return nullptr;
  }
  reinterpret_cast<double2 *>(slot)[0] = make_double2(v0, v1);
  reinterpret_cast<double2 *>(slot)[1] = make_double2(v2, v3);
  return blk;
}

__device__ __forceinline__ void bulk_add32(double *blk, const double *slot) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(slot);
  asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], 32;" ::"l"(blk), "r"(sa)
               : "memory");
}

// Drop-in mode: element `el`'s 2x2 block added at the reference map's offset
// (accumulate-into contract; elements of one launch share blocks), one 32-byte bulk
// reduction when the block address is 16-byte aligned, else four FP64 atomics.
template <int P>
__device__ __forceinline__ void frag_add_mapped(const Out &O, int el, int a, int b, int which, double kxx,
                                                double kxy, double kyx, double kyy, double *slot) {
  constexpr int NN = Dims<P>::NN;
  const int r0 = which ? b : a, c0 = which ? a : b;
  const double v0 = kxx, v1 = which ? kyx : kxy, v2 = which ? kxy : kyx, v3 = kyy;
  double *blk = O.mat + O.map[(el * NN + r0) * NN + c0];
  if ((reinterpret_cast<uintptr_t>(blk) & 15u) == 0) {
    reinterpret_cast<double2 *>(slot)[0] = make_double2(v0, v1);
    reinterpret_cast<double2 *>(slot)[1] = make_double2(v2, v3);
    const unsigned sa = (unsigned)__cvta_generic_to_shared(slot);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], 32;" ::"l"(blk), "r"(sa)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  } else {
    atomicAdd(blk + 0, v0);
    atomicAdd(blk + 1, v1);
    atomicAdd(blk + 2, v2);
    atomicAdd(blk + 3, v3);
  }
}

// The element pairs a warp assembles, in order.
struct PairCursor {
  int mesh;
  int ne;  // 0 ends the warp's loop
  int64_t k0;
  int tile = -1;      // dependency-ordered launches: the pair's tile
  bool last = false;  // ... and whether it is the tile's last pair
};

// Single mesh: pairs p, p + stride, ... of list positions [begin, end).
struct PairStride {
  static constexpr bool kBatched = false, kSched = false;
  int64_t begin, end, p, stride;
  __device__ PairCursor next(int) {
    PairCursor c{0, 0, begin + 2 * p};
    if (c.k0 < end) c.ne = (int)min((int64_t)2, end - c.k0);
    p += stride;
    return c;
  }
};

// One mesh, up to kMaxRanges list-position ranges of one launch (the band-split
// launches of fem_plan_assemble_host that share a schedule step): pairs p, p +
// stride, ... of their concatenation; a pair never straddles two ranges.
struct PairRanges {
  static constexpr bool kBatched = false, kSched = false;
  RangeList r;
  int64_t p, stride;
  __device__ PairCursor next(int) {
    PairCursor c{0, 0, 0};
    int64_t q = p;
    for (int i = 0; i < r.n; i++) {
      const int64_t np = (r.count[i] + 1) / 2;
      if (q < np) {
        c.k0 = r.begin[i] + 2 * q;
        c.ne = (int)min((int64_t)2, r.begin[i] + r.count[i] - c.k0);
        break;
      }
      q -= np;
    }
    p += stride;
    return c;
  }
};

// Many meshes: the pairs of the tiles this warp pulls from the launch's queue
// (one atomic counter per launch; tiles hold even element counts except at the
// end of a colour range, so pairs never straddle tiles).
struct PairQueue {
  static constexpr bool kBatched = true, kSched = false;
  const Tile *tiles;
  int ntiles;
  int *counter;
  int mesh;
  int64_t pos, tend;
  bool done;
  // lane 0: the tile after the current one, taken one tile ahead so that the queue
  // atomic's latency (long behind a later colour's reductions in L2) is hidden
  int ahead = -1;
  __device__ PairCursor next(int lane) {
    PairCursor c{0, 0, 0};
    while (!done && pos >= tend) {
      int t = 0;
      if (lane == 0) {
        t = ahead < 0 ? atomicAdd(counter, 1) : ahead;
        ahead = t < ntiles ? atomicAdd(counter, 1) : ntiles;
      }
      t = __shfl_sync(0xffffffffu, t, 0);
      if (t >= ntiles) {
        done = true;
      } else {
        const Tile tl = tiles[t];
        mesh = tl.mesh;
        pos = tl.begin;
        tend = tl.begin + tl.count;
      }
    }
    if (done) return c;
    c.mesh = mesh;
    c.k0 = pos;
    c.ne = (int)min((int64_t)2, tend - pos);
    pos += 2;
    return c;
  }
};

__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits (one lane) until group g of the schedule has finished all its tiles.  The
// wait is bounded: after S.waitLimitNs (or 2^22 polls, should the timer stall) it
// counts itself in status[0] and returns, and once any wait has run out no later
// wait starts, so a launch whose dependencies can never be met still ends within
// about one limit.  The tile then writes regardless; the host reports the count.
__device__ __noinline__ void sched_wait(const SchedArgs *S, int g) {
  const int target = S->groupTiles[g] + (g == S->stallGroup ? 1 : 0);
  const int *done = S->status + 2 + g;
  if (ld_acquire_gpu(done) >= target) return;
  const unsigned long long t0 = global_ns();
  for (unsigned it = 0;; it++) {
    __nanosleep(100);
    if (ld_acquire_gpu(done) >= target) return;
    if (ld_acquire_gpu(S->status) != 0) return;
    if (global_ns() - t0 > (unsigned long long)S->waitLimitNs || it >= (1u << 22)) {
      atomicAdd(S->status, 1);
      return;
    }
  }
}

// Dependency-ordered: warps pull tiles in dispatch order from one counter
// (status[1]); one mesh, or (BATCHED) the tiles of many meshes of one order, each
// tile naming its mesh.  Before the first write of a tile's pairs the warp waits for the
// groups its tile's group depends on (acquire); after the last pair of a tile it
// completes its writes -- the asynchronous bulk reductions included -- and counts
// the tile in its group (release).  A warp holds at most the tiles it has pulled,
// in dispatch order, and every dependency of a tile is an earlier group, so the
// earliest unfinished tile can always proceed: no wait is circular, whether or not
// every CTA of the grid is resident.
template <bool BATCHED>
struct PairSchedT {
  static constexpr bool kBatched = BATCHED, kSched = true;
  const SchedArgs *S;  // the kernel's __grid_constant__ parameter
  int tile = -1, held = -1, mesh = 0;
  int64_t pos = 0, tend = 0;
  bool done = false;
  __device__ PairCursor next(int lane) {
    PairCursor c{0, 0, 0};
    while (!done && pos >= tend) {
      int t = 0;
      if (lane == 0) t = atomicAdd(S->status + 1, 1);
      t = __shfl_sync(0xffffffffu, t, 0);
      if (t >= S->ntiles) {
        done = true;
      } else {
        const SchedTile tl = S->tiles[t];
        tile = t;
        if (BATCHED) mesh = tl.mesh;
        pos = tl.begin;
        tend = tl.begin + tl.count;
      }
    }
    if (done) return c;
    c.mesh = mesh;
    c.k0 = pos;
    c.ne = (int)min((int64_t)2, tend - pos);
    c.tile = tile;
    pos += 2;
    c.last = pos >= tend;
    return c;
  }
  __device__ void acquire(const PairCursor &c, int lane) {
    if (c.tile == held) return;
    held = c.tile;
    if (lane == 0) {
      const int g = S->tiles[c.tile].group;
      for (int i = S->depPtr[g]; i < S->depPtr[g + 1]; i++) sched_wait(S, S->deps[i]);
      __threadfence();
    }
    __syncwarp();
    // later bulk reductions (async proxy) are ordered after what the wait observed
    asm volatile("fence.proxy.async.global;" ::: "memory");
  }
  __device__ void release(const PairCursor &c, int lane) {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __threadfence();
    __syncwarp();
    if (lane == 0) atomicAdd(S->status + 2 + S->tiles[c.tile].group, 1);
  }
};
using PairSched = PairSchedT<false>;

// One warp's assembly loop over the pairs its generator yields.  `single` is the
// single-mesh kernel's argument block; batched generators read meshes[c.mesh].
template <int P, int MODE, typename Gen>
__device__ __forceinline__ void frag_loop(unsigned char *smem, Gen &gen, const AsmArgs &single,
                                          const AsmArgs *__restrict__ meshes) {
  constexpr bool PLAN = (MODE & kPlan) != 0;
  constexpr bool NL = (MODE & kNL) != 0;
  constexpr bool B16 = (MODE & kB16) != 0;  // BF16x6 element stiffness
  using F = FragDims<P>;
  using L = FragLayout<P, !PLAN, NL, B16, (MODE & kJac) != 0>;
  constexpr int NN = F::NN, NQ = F::NQ, K4 = F::K4, NTN = F::NTN, NQP = F::NQP, CS = F::CS;
  constexpr int STG = L::CS;  // staged bytes per element: plan code record or map rows
  constexpr bool RES = (MODE & kRes) != 0, JAC = (MODE & kJac) != 0;
  constexpr bool RUNS = (P == 3);  // order 3: staged row runs, one bulk reduction per adjacent run
  static_assert(!NL || !F::IL, "NONLINEAR strain: orders 2 and 3");
  static_assert(PLAN || !Gen::kBatched, "drop-in mode assembles one mesh");
  static_assert(!B16 || (!NL && P == 3), "BF16x6 stiffness: LINEAR, order 3");

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int e_ld = g >> 2, c_ld = g & 3;  // element / component this lane gathers
  const double *tabJ = reinterpret_cast<const double *>(smem + L::tabJ);
  const double2 *tabF = reinterpret_cast<const double2 *>(smem + L::tabF);
  const double *wqs = reinterpret_cast<const double *>(smem + L::wq);
  const double2 *csum = reinterpret_cast<const double2 *>(smem + L::csum);
  const double2 *tabB = reinterpret_cast<const double2 *>(smem + L::tabB);
  unsigned char *ws = smem + L::warps + warp * L::warp_bytes;
  double2 *WI0 = reinterpret_cast<double2 *>(ws + L::WI0);
  double2 *WI1 = reinterpret_cast<double2 *>(ws + L::WI1);
  double2 *WS0 = reinterpret_cast<double2 *>(ws + L::WS0);
  double2 *WS1 = reinterpret_cast<double2 *>(ws + L::WS1);
  double *SGs = reinterpret_cast<double *>(ws + L::SG);
  int *nid = reinterpret_cast<int *>(ws + L::NID);
  int *rb = reinterpret_cast<int *>(ws + L::RB);
  unsigned char *stage = ws + L::STAGE;
  double *redsW = reinterpret_cast<double *>(ws + L::REDS);  // staging slot s at redsW + 128 s
  double *ATs = reinterpret_cast<double *>(ws + L::AT);      // NONLINEAR tangent

  // Mesh arguments are read through `mtab` (for one mesh, a pointer to the kernel
  // parameter).  At p = 4 it is laundered once per step: the compiler then reloads
  // the arguments where they are used instead of hoisting ~20 loop-invariant values
  // into registers for the whole loop, which pushed the residual + Jacobian kernel
  // into 400 bytes of spills (3.4 against 3.0 ms on a 512^2 mesh).  At p = 2 the
  // reloads cost more than they save (1.80 against 1.60 ms on the annulus).
  const AsmArgs *mtab = meshes;
  auto args = [&](const PairCursor &c) -> const AsmArgs & {
    if constexpr (Gen::kBatched) {
      return mtab[c.mesh];
    } else {
      return *mtab;
    }
  };
  // node ids (two pairs ahead) and coordinate/state values (one pair ahead)
  int nodeA[K4], nodeB[K4], rbB[K4];
  double valB[K4];
  auto load_nodes = [&](const PairCursor &c, int *node) {
#pragma unroll
    for (int ks = 0; ks < K4; ks++) {
      const int a = 4 * ks + t;
      if constexpr (PLAN) {
        node[ks] = (e_ld < c.ne && a < NN) ? __ldg(args(c).connList + (c.k0 + e_ld) * NN + a) : -1;
      } else {
        node[ks] = (e_ld < c.ne && a < NN) ? __ldg(args(c).conn + __ldg(args(c).connPtr + c.k0 + e_ld) + a) : -1;
      }
    }
  };
  auto load_values = [&](const PairCursor &c, const int *node, double *val, int *rbv) {
#pragma unroll
    for (int ks = 0; ks < K4; ks++) {
      val[ks] = 0.0;
      rbv[ks] = 0;
      if (node[ks] >= 0) {
        const AsmArgs &M = args(c);
        const double *src = c_ld < 2 ? M.coords : M.states;
        val[ks] = __ldg(src + 2 * (int64_t)node[ks] + (c_ld & 1));
        if (PLAN && JAC && c_ld == 1) rbv[ks] = __ldg(M.rowp + node[ks]);
      }
    }
  };
  auto stage_codes = [&](const PairCursor &c, int buf) {
    if (c.ne > 0) {
      unsigned char *dst = stage + buf * 2 * STG;
      if constexpr (PLAN) {
        const unsigned char *src = args(c).blockCode + c.k0 * CS;
        for (int i = lane; i < c.ne * CS / 16; i += 32) cp_async16(dst + 16 * i, src + 16 * i);
      } else if constexpr (JAC) {
        // element map rows: 16-byte copies when a row set is a multiple of 16 bytes
        const int *src = args(c).map + c.k0 * NN * NN;
        if ((NN * NN) % 4 == 0 && (reinterpret_cast<uintptr_t>(src) & 15u) == 0) {
          for (int i = lane; i < c.ne * NN * NN / 4; i += 32) cp_async16(dst + 16 * i, src + 4 * i);
        } else {
          for (int i = lane; i < c.ne * NN * NN; i += 32) cp_async4(dst + 4 * i, src + i);
        }
      }
    }
    cp_async_commit();
  };

  // a grid launched after this one with programmatic serialization may start its CTAs
  // as this one's retire; it waits (griddepcontrol.wait) before it writes
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  bool dep_ready = false;
  PairCursor cur = gen.next(lane);
  PairCursor nxt = gen.next(lane);
  load_nodes(cur, nodeB);
  load_values(cur, nodeB, valB, rbB);
  load_nodes(nxt, nodeA);
  stage_codes(cur, 0);
  int buf = 0;

  for (; cur.ne > 0; buf ^= 1) {
    if constexpr (P == 4) asm volatile("" : "+l"(mtab));
    const int ne = cur.ne;
    const AsmArgs &M = args(cur);
    const double mu = M.mu, lam = M.lam, thick = M.t, c11 = lam + 2.0 * mu;
    // 0. commit this pair's gathered data
    double val[K4];
#pragma unroll
    for (int ks = 0; ks < K4; ks++) {
      val[ks] = valB[ks];
      const int a = 4 * ks + t;
      if (nodeB[ks] >= 0) {
        if (c_ld == 0) nid[e_ld * NN + a] = nodeB[ks];
        if (PLAN && JAC && c_ld == 1) rb[e_ld * NN + a] = rbB[ks];
      }
    }
    cp_async_wait_all();
    __syncwarp();
    // issue the following pairs' loads
    const PairCursor nn2 = gen.next(lane);
    stage_codes(nxt, buf ^ 1);
#pragma unroll
    for (int ks = 0; ks < K4; ks++) nodeB[ks] = nodeA[ks];
    load_values(nxt, nodeB, valB, rbB);
    load_nodes(nn2, nodeA);

    // 1. J stage: cj[tn] = (d/dxi, d/deta) of component c_ld of element e_ld at q = 4tn + t.
    //    J = sum_a x_a dN_a cancels by ~h/|x| (1e-4 on a 10x10 square of 1024^2
    //    elements), so the coordinates enter relative to the element's node 0 (an
    //    exact subtraction for nearby values) and x_0 sum_a dN_a is added back: the
    //    same sum, evaluated without the cancellation.
    const double xn0 = __shfl_sync(0xffffffffu, val[0], lane & ~3);
    const double x0 = c_ld < 2 ? xn0 : 0.0;
#pragma unroll
    for (int ks = 0; ks < K4; ks++) val[ks] -= x0;
    constexpr int TG = F::TG;
    double cj[4 * TG][2];
#pragma unroll
    for (int tn = 0; tn < 4 * TG; tn++) cj[tn][0] = cj[tn][1] = 0.0;
#pragma unroll
    for (int ks = 0; ks < K4; ks++)
#pragma unroll
      for (int tn = 0; tn < K4; tn++) dmma(cj[tn][0], cj[tn][1], val[ks], tabJ[(ks * K4 + tn) * 32 + lane]);
#pragma unroll
    for (int tn = 0; tn < K4; tn++) {
      const double2 cs = csum[4 * tn + t];
      cj[tn][0] = fma(x0, cs.x, cj[tn][0]);
      cj[tn][1] = fma(x0, cs.y, cj[tn][1]);
    }

    // 2. transpose, per group m of four column tiles: this lane takes quadrature
    //    point q = 4(4m + c_ld) + t of element e_ld
#pragma unroll
    for (int m = 0; m < TG; m++) {
      double rv[4][2];
      rv[0][0] = sel4(cj[4 * m][0], cj[4 * m + 1][0], cj[4 * m + 2][0], cj[4 * m + 3][0], c_ld);
      rv[0][1] = sel4(cj[4 * m][1], cj[4 * m + 1][1], cj[4 * m + 2][1], cj[4 * m + 3][1], c_ld);
#pragma unroll
      for (int r = 1; r < 4; r++) {
        const int src = c_ld ^ r;
        const double s0 = sel4(cj[4 * m][0], cj[4 * m + 1][0], cj[4 * m + 2][0], cj[4 * m + 3][0], src);
        const double s1 = sel4(cj[4 * m][1], cj[4 * m + 1][1], cj[4 * m + 2][1], cj[4 * m + 3][1], src);
        rv[r][0] = __shfl_xor_sync(0xffffffffu, s0, r << 2);
        rv[r][1] = __shfl_xor_sync(0xffffffffu, s1, r << 2);
      }
      // component k of this quadrature point came from round k ^ c_ld
      auto comp = [&](int k, int d) {
        const int r = k ^ c_ld;
        return d == 0 ? sel4(rv[0][0], rv[1][0], rv[2][0], rv[3][0], r)
                      : sel4(rv[0][1], rv[1][1], rv[2][1], rv[3][1], r);
      };
      const int tq = 4 * m + c_ld;  // column tile of this lane's quadrature point
      const int q = 4 * tq + t;
      const bool valid = e_ld < ne && tq < K4 && q < NQ;
      double2 wi0 = make_double2(0, 0), wi1 = make_double2(0, 0), ws0 = make_double2(0, 0), ws1 = make_double2(0, 0);
      double sg = 0.0;
      if (valid) {
        const double j00 = comp(0, 0), j01 = comp(0, 1), j10 = comp(1, 0), j11 = comp(1, 1);
        const double g00 = comp(2, 0), g01 = comp(2, 1), g10 = comp(3, 0), g11 = comp(3, 1);
        const double det = j00 * j11 - j01 * j10;
        const double inv = 1.0 / det;
        const double i00 = j11 * inv, i01 = -j01 * inv, i10 = -j10 * inv, i11 = j00 * inv;
        const double st = wqs[q] * det * thick;
        const double rs = sqrt(fabs(st));
        sg = st < 0.0 ? -1.0 : 1.0;
        const double sw = sg * rs;
        const double uxx = g00 * i00 + g01 * i10, uxy = g00 * i01 + g01 * i11;
        const double uyx = g10 * i00 + g11 * i10, uyy = g10 * i01 + g11 * i11;
        wi0 = make_double2(rs * i00, rs * i10);
        wi1 = make_double2(rs * i01, rs * i11);
        if constexpr (NL) {
          // Green strain E = 1/2 (g + g^T + g^T g), S = 2 mu E + lam tr(E) I, first Piola
          // P = F S (F = I + g); tangent A_{il,kn} = delta_ik S_ln + mu F_in F_kl
          // + mu (F F^T)_ik delta_ln + lam F_il F_kn (element/FEKernels.h:286-315,
          // NONLINEAR), stored times sign(s) as [l][i][k][n]
          const double F[2][2] = {{1.0 + uxx, uxy}, {uyx, 1.0 + uyy}};
          const double e00 = 0.5 * (2.0 * uxx + uxx * uxx + uyx * uyx);
          const double e01 = 0.5 * (uxy + uyx + uxx * uxy + uyx * uyy);
          const double e11 = 0.5 * (2.0 * uyy + uxy * uxy + uyy * uyy);
          const double trE = e00 + e11;
          const double Sm[2][2] = {{2.0 * mu * e00 + lam * trE, 2.0 * mu * e01}, {2.0 * mu * e01, 2.0 * mu * e11 + lam * trE}};
          const double pxx = F[0][0] * Sm[0][0] + F[0][1] * Sm[1][0], pxy = F[0][0] * Sm[0][1] + F[0][1] * Sm[1][1];
          const double pyx = F[1][0] * Sm[0][0] + F[1][1] * Sm[1][0], pyy = F[1][0] * Sm[0][1] + F[1][1] * Sm[1][1];
          ws0 = make_double2(sw * pxx, sw * pyx);  // (P-hat_x0, P-hat_y0)
          ws1 = make_double2(sw * pxy, sw * pyy);  // (P-hat_x1, P-hat_y1)
          if (JAC && tq < K4) {
            double *at = ATs + (e_ld * NQP + q) * 16;
#pragma unroll
            for (int ll = 0; ll < 2; ll++)
#pragma unroll
              for (int ii2 = 0; ii2 < 2; ii2++)
#pragma unroll
                for (int kk = 0; kk < 2; kk++) {
                  double v2[2];
#pragma unroll
                  for (int nn = 0; nn < 2; nn++) {
                    const double bik = F[ii2][0] * F[kk][0] + F[ii2][1] * F[kk][1];
                    double v = mu * F[ii2][nn] * F[kk][ll] + lam * F[ii2][ll] * F[kk][nn];
                    if (ii2 == kk) v += Sm[ll][nn];
                    if (ll == nn) v += mu * bik;
                    v2[nn] = sg * v;
                  }
                  *reinterpret_cast<double2 *>(at + ll * 8 + ii2 * 4 + kk * 2) = make_double2(v2[0], v2[1]);
                }
          }
        } else {
          const double tr = uxx + uyy;
          const double sxx = sw * (2.0 * mu * uxx + lam * tr);
          const double sxy = sw * (mu * (uxy + uyx));
          const double syy = sw * (2.0 * mu * uyy + lam * tr);
          ws0 = make_double2(sxx, sxy);
          ws1 = make_double2(sxy, syy);
        }
      } else if (NL && JAC && tq < K4) {
        double2 *at = reinterpret_cast<double2 *>(ATs + (e_ld * NQP + q) * 16);
#pragma unroll
        for (int j = 0; j < 8; j++) at[j] = make_double2(0.0, 0.0);
      }
      if (tq < K4) {
        const int o = e_ld * NQP + q;
        WI0[o] = wi0;
        WI1[o] = wi1;
        WS0[o] = ws0;
        WS1[o] = ws1;
        SGs[o] = sg;
      }
    }
    __syncwarp();

    // the warp's first writes wait for the grid launched before this one (programmatic
    // dependent launch: its gathers and element arithmetic ran while that grid drained)
    if (!dep_ready) {
      asm volatile("griddepcontrol.wait;" ::: "memory");
      dep_ready = true;
    }
    if constexpr (Gen::kSched) gen.acquire(cur, lane);
    const Out O{M.mat, M.residual, stage + buf * 2 * STG, rb, reinterpret_cast<const int *>(stage + buf * 2 * STG)};
    if constexpr (!F::IL) {
      // node tiles on the tensor cores: both at p = 3; at p = 2 only tile 0 (nodes 0-7),
      // node 8 (alone in tile 1) has its row and column on the FP64 pipe (12 instead of
      // 36 MMAs per element)
      constexpr int NTM = (P == 2) ? 1 : NTN;
      constexpr int NPAIR = NTM * (NTM + 1) / 2;
      const int pa = 4 * (g & 1) + (g >> 1);  // pi(g)
      for (int el = 0; el < ne; el++) {
        // pair layout: the first element's residual writes before the second's
        if (PLAN && el > 0) __syncwarp();
        if constexpr (B16) {
          // BF16x6 element stiffness: M_ij = sum_q s G_i(q, a) G_j(q, b) as m16n8k16
          // products (k = quadrature points 0-15; rows a and columns b of the two node
          // tiles, a = 8h + pi(g) and b = 8h' + pi(n)); each FP64 operand is split into
          // three BF16 parts and six part products accumulate in FP32 (hi*hi, hi*mid,
          // mid*hi, hi*lo, lo*hi, mid*mid: ~FP32 accuracy; the two-way BF16x3 split
          // leaves ~4e-6 relative error in K).  Lane (g, t) holds the values of the
          // quadrature points q_k = 2t + (k & 1) + 8 (k >> 1) of nodes 8h + pi(g).
          double gv[2][4][2];  // [i][k][h]: G-hat_i(q_k, 8h + pi(g)) = sqrt|s| (dN J^-1)_i
          double sgk[4];
          double rx[2] = {0.0, 0.0}, ry[2] = {0.0, 0.0};
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const int q = 2 * t + (k & 1) + 8 * (k >> 1);
            const int o = el * NQP + q;
            const bool qv = q < NQ;
            const double2 w0 = qv ? WI0[o] : make_double2(0.0, 0.0), w1 = qv ? WI1[o] : make_double2(0.0, 0.0);
            sgk[k] = qv ? SGs[o] : 0.0;
            double2 s0 = make_double2(0.0, 0.0), s1 = make_double2(0.0, 0.0);
            if (RES && qv) {
              s0 = WS0[o];
              s1 = WS1[o];
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const double2 d = tabB[(2 * k + h) * 32 + lane];
              gv[0][k][h] = fma(w0.x, d.x, w0.y * d.y);
              gv[1][k][h] = fma(w1.x, d.x, w1.y * d.y);
              if constexpr (RES) {
                rx[h] = fma(gv[0][k][h], s0.x, fma(gv[1][k][h], s1.x, rx[h]));
                ry[h] = fma(gv[0][k][h], s0.y, fma(gv[1][k][h], s1.y, ry[h]));
              }
            }
          }
          if constexpr (RES) {
            // sum over the four lanes t of node 8h + pi(g); lane t = h writes it
#pragma unroll
            for (int h = 0; h < 2; h++) {
              rx[h] += __shfl_xor_sync(0xffffffffu, rx[h], 1);
              ry[h] += __shfl_xor_sync(0xffffffffu, ry[h], 1);
              rx[h] += __shfl_xor_sync(0xffffffffu, rx[h], 2);
              ry[h] += __shfl_xor_sync(0xffffffffu, ry[h], 2);
            }
            const int a = 8 * t + pa;
            if (t < 2 && a < NN) {
              const double sx = t ? rx[1] : rx[0], sy = t ? ry[1] : ry[0];
              double *dst = M.residual + 2 * (int64_t)nid[el * NN + a];
              if (PLAN && O.codes[el * CS + NN * NN + a]) {
                *reinterpret_cast<double2 *>(dst) = make_double2(sx, sy);
              } else {
                atomicAdd(dst, sx);
                atomicAdd(dst + 1, sy);
              }
            }
          }
          if constexpr (JAC) {
            // split operands: B[part][j][h][r] (column node 8h + pi(g)), A = sign(s) B
            // packed as row fragments: A[part][i][r] (rows pi(g), 8 + pi(g))
            uint32_t pb[3][2][4][2];  // [part][i][k][h] raw BF16 bits
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
              for (int k = 0; k < 4; k++)
#pragma unroll
                for (int h = 0; h < 2; h++) split3(gv[i][k][h], pb[0][i][k][h], pb[1][i][k][h], pb[2][i][k][h]);
            uint32_t Af[3][2][4], Bf[3][2][2][2];
#pragma unroll
            for (int pt = 0; pt < 3; pt++)
#pragma unroll
              for (int i = 0; i < 2; i++) {
                auto sv = [&](int k, int h) { return pb[pt][i][k][h] ^ (sgk[k] < 0.0 ? 0x8000u : 0u); };
                Af[pt][i][0] = sv(0, 0) | (sv(1, 0) << 16);
                Af[pt][i][1] = sv(0, 1) | (sv(1, 1) << 16);
                Af[pt][i][2] = sv(2, 0) | (sv(3, 0) << 16);
                Af[pt][i][3] = sv(2, 1) | (sv(3, 1) << 16);
#pragma unroll
                for (int h = 0; h < 2; h++) {
                  Bf[pt][i][h][0] = pb[pt][i][0][h] | (pb[pt][i][1][h] << 16);
                  Bf[pt][i][h][1] = pb[pt][i][2][h] | (pb[pt][i][3][h] << 16);
                }
              }
            float acc[2][2][2][4];  // [i][j][h (column tile)][c]
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
              for (int j = 0; j < 2; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
#pragma unroll
                  for (int c = 0; c < 4; c++) acc[i][j][h][c] = 0.0f;
                  // smallest terms first
                  bmma(acc[i][j][h], Af[2][i], Bf[0][j][h][0], Bf[0][j][h][1]);
                  bmma(acc[i][j][h], Af[0][i], Bf[2][j][h][0], Bf[2][j][h][1]);
                  bmma(acc[i][j][h], Af[1][i], Bf[1][j][h][0], Bf[1][j][h][1]);
                  bmma(acc[i][j][h], Af[1][i], Bf[0][j][h][0], Bf[0][j][h][1]);
                  bmma(acc[i][j][h], Af[0][i], Bf[1][j][h][0], Bf[1][j][h][1]);
                  bmma(acc[i][j][h], Af[0][i], Bf[0][j][h][0], Bf[0][j][h][1]);
                }
            // lane (g, t): c = 2 r + u holds M_ij[a = 8r + pi(g)][b = 8h + 4u + t]: whole
            // 2x2 blocks, four consecutive columns across the lanes t.  Blocks to add go
            // to the staging slots of the FP64 layout (node-tile pair (r, h) = (TA, TB);
            // the pair (1, 0) is the transposed half of (0, 1)) and leave as row runs.
            asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
            __syncwarp();
#pragma unroll
            for (int r = 0; r < 2; r++)
#pragma unroll
              for (int h = 0; h < 2; h++)
#pragma unroll
                for (int u = 0; u < 2; u++) {
                  const int a = 8 * r + pa, b = 8 * h + 4 * u + t, c = 2 * r + u;
                  if (a < NN && b < NN) {
                    const double mxx = acc[0][0][h][c], mxy = acc[0][1][h][c];
                    const double myx = acc[1][0][h][c], myy = acc[1][1][h][c];
                    const double kxx = c11 * mxx + mu * myy, kxy = lam * mxy + mu * myx;
                    const double kyx = lam * myx + mu * mxy, kyy = c11 * myy + mu * mxx;
                    const int sl = (r == 1 && h == 0) ? frag_slot(1, g & 1, 1) : frag_slot(r + h, u, 0);
                    const int pos = (r == 1 && h == 0) ? 8 * (g >> 1) + 4 * u + t : 4 * g + t;
                    frag_put<P, PLAN>(O, el, a, b, 0, kxx, kxy, kyx, kyy, redsW + 128 * sl + 4 * pos);
                  }
                }
            if (PLAN && el > 0) pair_first_landed();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (PLAN && el > 0) pair_first_visible();
#pragma unroll
            for (int v = 0; v < 2; v++) {
              const int run = lane + 32 * v;
              frag_issue_run<P, PLAN>(O, el, run >> 3, run & 7, redsW);
            }
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          }
          continue;
        }
        // 3.-5. quadrature k-steps outermost: per step each lane forms its fragments
        // G-hat_i(q = 4ks + t, a = 8T + pi(g)), adds its residual partials and issues
        // the 4 NPAIR independent stiffness MMAs of all node-tile pairs
        double acc[NPAIR][4][2];
        double rp[NTN][2];
        double n8[4] = {0.0, 0.0, 0.0, 0.0}, d8[4] = {0.0, 0.0, 0.0, 0.0};  // p = 2: M[8][pi(g)], M[8][8]
  #pragma unroll
        for (int k = 0; k < NPAIR; k++)
  #pragma unroll
          for (int c = 0; c < 4; c++) acc[k][c][0] = acc[k][c][1] = 0.0;
  #pragma unroll
        for (int T = 0; T < NTN; T++) rp[T][0] = rp[T][1] = 0.0;
  #pragma unroll
        for (int ks = 0; ks < K4; ks++) {
          const int o = el * NQP + 4 * ks + t;
          const double2 w0 = WI0[o], w1 = WI1[o];
          const double sg = SGs[o];
          double fr[NTN][2];
  #pragma unroll
          for (int T = 0; T < NTN; T++) {
            const double2 d = tabF[(ks * NTN + T) * 32 + lane];
            fr[T][0] = fma(w0.x, d.x, w0.y * d.y);
            fr[T][1] = fma(w1.x, d.x, w1.y * d.y);
          }
          if constexpr (RES) {
            const double2 s0 = WS0[o], s1 = WS1[o];
  #pragma unroll
            for (int T = 0; T < NTN; T++) {
              rp[T][0] = fma(fr[T][0], s0.x, fma(fr[T][1], s1.x, rp[T][0]));
              rp[T][1] = fma(fr[T][0], s0.y, fma(fr[T][1], s1.y, rp[T][1]));
            }
          }
          if constexpr (JAC && NL) {
            // K_ik[a][b] = sum over (q, l) of G-hat_l(q, a) B_ikl(q, b),
            // B_ikl = sign(s) sum_n A_{il,kn} G-hat_n(q, b): 4 (i, k) x 2 (l) MMAs per pair
            const double *at = ATs + o * 16;
            double h0 = 0.0, h1 = 0.0;
            if constexpr (P == 2) {
              h0 = __shfl_sync(0xffffffffu, fr[1][0], t);
              h1 = __shfl_sync(0xffffffffu, fr[1][1], t);
            }
#pragma unroll
            for (int ll = 0; ll < 2; ll++) {
              double C[2][2][2];  // [i][k][n]
#pragma unroll
              for (int j = 0; j < 4; j++) {
                const double2 v = *reinterpret_cast<const double2 *>(at + ll * 8 + 2 * j);
                C[j >> 1][j & 1][0] = v.x;
                C[j >> 1][j & 1][1] = v.y;
              }
              int k = 0;
#pragma unroll
              for (int TA = 0; TA < NTM; TA++) {
#pragma unroll
                for (int TB = TA; TB < NTM; TB++, k++) {
#pragma unroll
                  for (int ik = 0; ik < 4; ik++) {
                    const double bv = fma(C[ik >> 1][ik & 1][0], fr[TB][0], C[ik >> 1][ik & 1][1] * fr[TB][1]);
                    dmma(acc[k][ik][0], acc[k][ik][1], fr[TA][ll], bv);
                  }
                }
              }
              if constexpr (P == 2) {
                const double hl = ll ? h1 : h0;
#pragma unroll
                for (int ik = 0; ik < 4; ik++) {
                  n8[ik] = fma(hl, fma(C[ik >> 1][ik & 1][0], fr[0][0], C[ik >> 1][ik & 1][1] * fr[0][1]), n8[ik]);
                  d8[ik] = fma(hl, fma(C[ik >> 1][ik & 1][0], h0, C[ik >> 1][ik & 1][1] * h1), d8[ik]);
                }
              }
            }
          }
          if constexpr (JAC && P == 2 && !NL) {
            // G-hat_i(q, 8) sits in lane (g = 0, t), tile 1
            const double h0 = __shfl_sync(0xffffffffu, fr[1][0], t), h1 = __shfl_sync(0xffffffffu, fr[1][1], t);
            const double s0 = sg * h0, s1 = sg * h1;
            n8[0] = fma(s0, fr[0][0], n8[0]);
            n8[1] = fma(s0, fr[0][1], n8[1]);
            n8[2] = fma(s1, fr[0][0], n8[2]);
            n8[3] = fma(s1, fr[0][1], n8[3]);
            d8[0] = fma(s0, h0, d8[0]);
            d8[1] = fma(s0, h1, d8[1]);
            d8[2] = fma(s1, h0, d8[2]);
            d8[3] = fma(s1, h1, d8[3]);
          }
          if constexpr (JAC && !NL) {
            int k = 0;
  #pragma unroll
            for (int TA = 0; TA < NTM; TA++) {
              const double a0 = sg * fr[TA][0], a1 = sg * fr[TA][1];
  #pragma unroll
              for (int TB = TA; TB < NTM; TB++, k++) {
                dmma(acc[k][0][0], acc[k][0][1], a0, fr[TB][0]);
                dmma(acc[k][1][0], acc[k][1][1], a0, fr[TB][1]);
                dmma(acc[k][2][0], acc[k][2][1], a1, fr[TB][0]);
                dmma(acc[k][3][0], acc[k][3][1], a1, fr[TB][1]);
              }
            }
          }
        }
        // residual: sum over the four lanes t of a node (reduce-scatter over node tiles)
        if constexpr (RES) {
          const int Tm = t >> 1, To = Tm ^ 1;
          double sx = (Tm ? rp[1][0] : rp[0][0]) + __shfl_xor_sync(0xffffffffu, To ? rp[1][0] : rp[0][0], 2);
          double sy = (Tm ? rp[1][1] : rp[0][1]) + __shfl_xor_sync(0xffffffffu, To ? rp[1][1] : rp[0][1], 2);
          sx += __shfl_xor_sync(0xffffffffu, sx, 1);
          sy += __shfl_xor_sync(0xffffffffu, sy, 1);
          const int a = 8 * Tm + pa;
          if ((t & 1) == 0 && a < NN) {
            double *dst = M.residual + 2 * (int64_t)nid[el * NN + a];
            if (PLAN && O.codes[el * CS + NN * NN + a]) {
              *reinterpret_cast<double2 *>(dst) = make_double2(sx, sy);
            } else {
              atomicAdd(dst, sx);
              atomicAdd(dst + 1, sy);
            }
          }
        }
        // stiffness blocks, order 3: lane (g, t) holds (a = 8TA + pi(g), b = 8TB + 4h + t).  Blocks that
        // are added (drop-in: all; plan: later colours) are staged so that each row run of
        // four consecutive columns is contiguous in shared memory -- slot s = (pair, h,
        // direct/transposed), direct position 4g + t (row a, columns 8TB + 4h + 0..3),
        // transposed position 8t + pi(g) (row b, columns 8TA + 4*half + 0..3) -- and then
        // reduced with one 128-byte bulk operation per run whose four blocks are adjacent in
        // the matrix, else one 32-byte operation per block.
        if constexpr (JAC && RUNS) {
          // every lane's previous bulk reads of the staging slots are complete
          asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          __syncwarp();
          int k = 0;
  #pragma unroll
          for (int TA = 0; TA < NTN; TA++) {
  #pragma unroll
            for (int TB = TA; TB < NTN; TB++, k++) {
              const int a = 8 * TA + pa;
  #pragma unroll
              for (int h = 0; h < 2; h++) {
                const int b = 8 * TB + 4 * h + t;
                if (a < NN && b < NN) {
                  const double mxx = acc[k][0][h], mxy = acc[k][1][h], myx = acc[k][2][h], myy = acc[k][3][h];
                  // LINEAR: plane-stress combination of M; NONLINEAR: the block itself
                  const double kxx = NL ? mxx : c11 * mxx + mu * myy;
                  const double kxy = NL ? mxy : lam * mxy + mu * myx;
                  const double kyx = NL ? myx : lam * myx + mu * mxy;
                  const double kyy = NL ? myy : c11 * myy + mu * mxx;
                  const int s0 = frag_slot(k, h, 0);
                  if (TA < TB) {
                    const int s1 = frag_slot(k, h, 1);
                    frag_put<P, PLAN>(O, el, a, b, 0, kxx, kxy, kyx, kyy, redsW + 128 * s0 + 4 * (4 * g + t));
                    frag_put<P, PLAN>(O, el, a, b, 1, kxx, kxy, kyx, kyy, redsW + 128 * s1 + 4 * (8 * t + pa));
                  } else if (!NL) {
                    frag_put<P, PLAN>(O, el, a, b, 0, kxx, kxy, kyx, kyy, redsW + 128 * s0 + 4 * (4 * g + t));
                  } else if (a <= b) {
                    // NONLINEAR diagonal tile: (a, b) for a <= b and, for a < b, its exact
                    // transpose (b, a) at the staging position the (b, a) lane would use
                    frag_put<P, PLAN>(O, el, a, b, 0, kxx, kxy, kyx, kyy, redsW + 128 * s0 + 4 * (4 * g + t));
                    if (a < b) {
                      const int xb = b - 8 * TA, xa = a - 8 * TA;  // pi(g') = xb; a = 8T + 4h' + t'
                      const int gb = 2 * (xb & 3) + (xb >> 2);
                      const int st = frag_slot(k, xa >> 2, 0);
                      frag_put<P, PLAN>(O, el, a, b, 1, kxx, kxy, kyx, kyy, redsW + 128 * st + 4 * (4 * gb + (xa & 3)));
                    }
                  }
                }
              }
            }
          }
          if (PLAN && el > 0) pair_first_landed();
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (PLAN && el > 0) pair_first_visible();
          // 64 runs (8 slots x 8 runs), two per lane
  #pragma unroll
          for (int u = 0; u < 2; u++) {
            const int run = lane + 32 * u;
            frag_issue_run<P, PLAN>(O, el, run >> 3, run & 7, redsW);
          }
          asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
        // stiffness blocks, order 2 (plan, LINEAR): lane (g, t) writes (pi(g), 4h + t),
        // h = 0, 1, and lanes t < 2 / (g = 0, t = 2) a node-8 block; first stores go out
        // at once, the blocks to add are staged in slots 0-2 and leave after one proxy
        // fence, as one bulk group (a fence per block cost 5 % of the order-2 time)
        if constexpr (JAC && !RUNS && PLAN && !NL && P == 2) {
          if (el > 0) pair_order_fence();
          asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          double *reds = redsW + 4 * lane;
          double *dst[3] = {nullptr, nullptr, nullptr};
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const double mxx = acc[0][0][h], mxy = acc[0][1][h], myx = acc[0][2][h], myy = acc[0][3][h];
            const double kxx = c11 * mxx + mu * myy, kxy = lam * mxy + mu * myx;
            const double kyx = lam * myx + mu * mxy, kyy = c11 * myy + mu * mxx;
            dst[h] = frag_stage<P>(O, el, pa, 4 * h + t, 0, kxx, kxy, kyx, kyy, reds + 128 * h);
          }
#pragma unroll
          for (int c = 0; c < 4; c++) {
            n8[c] += __shfl_xor_sync(0xffffffffu, n8[c], 1);
            n8[c] += __shfl_xor_sync(0xffffffffu, n8[c], 2);
            d8[c] += __shfl_xor_sync(0xffffffffu, d8[c], 1);
            d8[c] += __shfl_xor_sync(0xffffffffu, d8[c], 2);
          }
          const bool diag = (g == 0 && t == 2);
          if (t < 2 || diag) {
            const double mxx = diag ? d8[0] : n8[0], mxy = diag ? d8[1] : n8[1];
            const double myx = diag ? d8[2] : n8[2], myy = diag ? d8[3] : n8[3];
            const double kxx = c11 * mxx + mu * myy, kxy = lam * mxy + mu * myx;
            const double kyx = lam * myx + mu * mxy, kyy = c11 * myy + mu * mxx;
            dst[2] = frag_stage<P>(O, el, 8, diag ? 8 : pa, diag ? 0 : t, kxx, kxy, kyx, kyy, reds + 128 * 2);
          }
          if (dst[0] || dst[1] || dst[2]) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
#pragma unroll
            for (int s2 = 0; s2 < 3; s2++)
              if (dst[s2]) bulk_add32(dst[s2], reds + 128 * s2);
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          }
        }
        // stiffness blocks, order 2 (drop-in or NONLINEAR): lane (g, t) holds
        // (a = 8TA + pi(g), b = 8TB + 4h + t), each written (or added) on its own
        if constexpr (JAC && !RUNS && !(PLAN && !NL && P == 2)) {
          if (PLAN && el > 0) pair_order_fence();
          asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          int k = 0, slot = 0;
          double *reds = redsW + 4 * lane;
  #pragma unroll
          for (int TA = 0; TA < NTM; TA++) {
  #pragma unroll
            for (int TB = TA; TB < NTM; TB++, k++) {
              const int a = 8 * TA + pa;
  #pragma unroll
              for (int h = 0; h < 2; h++) {
                const int b = 8 * TB + 4 * h + t;
                if (a < NN && b < NN) {
                  const double mxx = acc[k][0][h], mxy = acc[k][1][h], myx = acc[k][2][h], myy = acc[k][3][h];
                  // LINEAR: plane-stress combination of M; NONLINEAR: the block itself
                  const double kxx = NL ? mxx : c11 * mxx + mu * myy;
                  const double kxy = NL ? mxy : lam * mxy + mu * myx;
                  const double kyx = NL ? myx : lam * myx + mu * mxy;
                  const double kyy = NL ? myy : c11 * myy + mu * mxx;
                  // NONLINEAR diagonal tiles: (a, b) for a <= b and its exact transpose
                  const bool dir = TA < TB || !NL || a <= b;
                  const bool trn = TA < TB || (NL && a < b);
                  if constexpr (PLAN) {
                    if (dir) frag_write<P>(O, el, a, b, 0, kxx, kxy, kyx, kyy, reds + 128 * slot++);
                    if (trn) frag_write<P>(O, el, a, b, 1, kxx, kxy, kyx, kyy, reds + 128 * slot++);
                  } else {
                    if (dir) frag_add_mapped<P>(O, el, a, b, 0, kxx, kxy, kyx, kyy, reds + 128 * slot++);
                    if (trn) frag_add_mapped<P>(O, el, a, b, 1, kxx, kxy, kyx, kyy, reds + 128 * slot++);
                  }
                }
              }
            }
          }
          if constexpr (P == 2) {
            // node 8: sum the partials over the four lanes t; lane t = 0 writes (8, pi(g)),
            // t = 1 its transpose (pi(g), 8), lane (g = 0, t = 2) the diagonal block (8, 8)
#pragma unroll
            for (int c = 0; c < 4; c++) {
              n8[c] += __shfl_xor_sync(0xffffffffu, n8[c], 1);
              n8[c] += __shfl_xor_sync(0xffffffffu, n8[c], 2);
              d8[c] += __shfl_xor_sync(0xffffffffu, d8[c], 1);
              d8[c] += __shfl_xor_sync(0xffffffffu, d8[c], 2);
            }
            const bool diag = (g == 0 && t == 2);
            if (t < 2 || diag) {
              const double mxx = diag ? d8[0] : n8[0], mxy = diag ? d8[1] : n8[1];
              const double myx = diag ? d8[2] : n8[2], myy = diag ? d8[3] : n8[3];
              const double kxx = NL ? mxx : c11 * mxx + mu * myy;
              const double kxy = NL ? mxy : lam * mxy + mu * myx;
              const double kyx = NL ? myx : lam * myx + mu * mxy;
              const double kyy = NL ? myy : c11 * myy + mu * mxx;
              const int b = diag ? 8 : pa, w = diag ? 0 : t;
              if constexpr (PLAN) {
                frag_write<P>(O, el, 8, b, w, kxx, kxy, kyx, kyy, reds + 128 * slot);
              } else {
                frag_add_mapped<P>(O, el, 8, b, w, kxx, kxy, kyx, kyy, reds + 128 * slot);
              }
            }
          }
        }
      }
    } else {
      // interleaved rows r = 2a + i (p = 4): lane (g, t) builds G-hat_i(q = 4ks + t,
      // a = 4T + g/2), i = g%2, the A fragment of row tile T and the B fragment of
      // column tile T; lanes l and l^4 hold the two rows of a 2x2 block.  The stiffness
      // takes one pass per group of tile pairs; the residual rides on the first three
      // groups (a pass of its own when the Jacobian is not assembled).
      const int ii = g & 1, ah = g >> 1;
      const double2 *WIi = ii ? WI1 : WI0;
      const double2 *WSi = ii ? WS1 : WS0;
      double *reds = redsW + 4 * lane;
      int nw = 0;  // writes so far: ring position of the staging slot
      for (int el = 0; el < ne; el++) {
        if (PLAN && el > 0) pair_order_fence();
        // residual R_(a,i'): lane partials rp over its quadrature points (with the
        // Jacobian, accumulated by the first three stiffness groups, which between them
        // form every column tile's fragments; alone, in a pass of its own), then a full
        // sum over the component pair (xor 4) and a reduce-scatter over the four lanes
        // t (lane t ends with tiles 2t and 2t + 1)
        double rp[8][2];
#pragma unroll
        for (int T = 0; T < 8; T++) rp[T][0] = rp[T][1] = 0.0;
        auto res_write = [&]() {
#pragma unroll
          for (int T = 0; T < K4; T++)
#pragma unroll
            for (int c = 0; c < 2; c++) rp[T][c] += __shfl_xor_sync(0xffffffffu, rp[T][c], 4);
          const int hi = t >> 1, lo = t & 1;
          double w4[4][2], z[2][2];
#pragma unroll
          for (int k = 0; k < 4; k++)
#pragma unroll
            for (int c = 0; c < 2; c++)
              w4[k][c] = (hi ? rp[4 + k][c] : rp[k][c]) + __shfl_xor_sync(0xffffffffu, hi ? rp[k][c] : rp[4 + k][c], 2);
#pragma unroll
          for (int mm = 0; mm < 2; mm++)
#pragma unroll
            for (int c = 0; c < 2; c++)
              z[mm][c] = (lo ? w4[2 + mm][c] : w4[mm][c]) + __shfl_xor_sync(0xffffffffu, lo ? w4[mm][c] : w4[2 + mm][c], 1);
#pragma unroll
          for (int mm = 0; mm < 2; mm++) {
            const int a = 4 * (2 * t + mm) + ah;
            if (ii == 0 && a < NN) {
              double *dst = M.residual + 2 * (int64_t)nid[el * NN + a];
              if (PLAN && O.codes[el * CS + NN * NN + a]) {
                *reinterpret_cast<double2 *>(dst) = make_double2(z[mm][0], z[mm][1]);
              } else {
                atomicAdd(dst, z[mm][0]);
                atomicAdd(dst + 1, z[mm][1]);
              }
            }
          }
        };
        if constexpr (RES && !JAC) {
#pragma unroll
          for (int ks = 0; ks < K4; ks++) {
            const int o = el * NQP + 4 * ks + t;
            const double2 w = WIi[o];
            const double2 sj = WSi[o];  // (S-hat_xj, S-hat_yj), j = this lane's component
#pragma unroll
            for (int C = 0; C < K4; C++) {
              const double2 d = tabF[(ks * K4 + C) * 16 + 4 * ah + t];
              const double gv = fma(w.x, d.x, w.y * d.y);
              rp[C][0] = fma(gv, sj.x, rp[C][0]);
              rp[C][1] = fma(gv, sj.y, rp[C][1]);
            }
          }
          res_write();
        }
        // stiffness: the 28 tile pairs (R, C >= R) in four groups, each a triangle
        // {R0..R1-1}^2 or a rectangle {R0..R1-1} x {C0..C1-1} of the upper triangle
        // (at most ten live accumulator tiles); within a group the k-steps are
        // outermost and each fragment of the group's rows and columns is formed once
        // per step: 17 fragment builds per k-step for the 28 tile pairs
        auto group = [&](auto r0c, auto r1c, auto c0c, auto c1c, auto resc) {
          constexpr int R0 = decltype(r0c)::value, R1 = decltype(r1c)::value;
          constexpr int C0 = decltype(c0c)::value, C1 = decltype(c1c)::value;
          constexpr bool GRES = RES && decltype(resc)::value;  // residual tiles C0..C1-1
          double acc[R1 - R0][C1 - C0][2];
#pragma unroll
          for (int R = R0; R < R1; R++)
#pragma unroll
            for (int C = C0; C < C1; C++) acc[R - R0][C - C0][0] = acc[R - R0][C - C0][1] = 0.0;
#pragma unroll
          for (int ks = 0; ks < K4; ks++) {
            const int o = el * NQP + 4 * ks + t;
            const double2 w = WIi[o];
            const double sg = SGs[o];
            double fr[K4];
#pragma unroll
            for (int T = 0; T < K4; T++) {
              if ((T >= R0 && T < R1) || (T >= C0 && T < C1)) {
                const double2 d = tabF[(ks * K4 + T) * 16 + 4 * ah + t];
                fr[T] = fma(w.x, d.x, w.y * d.y);
              }
            }
            if constexpr (GRES) {
              const double2 sj = WSi[o];
#pragma unroll
              for (int C = C0; C < C1; C++) {
                rp[C][0] = fma(fr[C], sj.x, rp[C][0]);
                rp[C][1] = fma(fr[C], sj.y, rp[C][1]);
              }
            }
#pragma unroll
            for (int R = R0; R < R1; R++) {
              const double af = sg * fr[R];
#pragma unroll
              for (int C = (R > C0 ? R : C0); C < C1; C++)
                dmma(acc[R - R0][C - C0][0], acc[R - R0][C - C0][1], af, fr[C]);
            }
          }
          // blocks: lane pair (l, l^4) exchanges rows; lane i = 0 writes (a, b), lane
          // i = 1 writes (b, a) = (a, b)^T
#pragma unroll
          for (int R = R0; R < R1; R++) {
            const int a = 4 * R + ah;
#pragma unroll
            for (int C = (R > C0 ? R : C0); C < C1; C++) {
              const double o0 = __shfl_xor_sync(0xffffffffu, acc[R - R0][C - C0][0], 4);
              const double o1 = __shfl_xor_sync(0xffffffffu, acc[R - R0][C - C0][1], 4);
              const double mxx = ii ? o0 : acc[R - R0][C - C0][0], mxy = ii ? o1 : acc[R - R0][C - C0][1];
              const double myx = ii ? acc[R - R0][C - C0][0] : o0, myy = ii ? acc[R - R0][C - C0][1] : o1;
              const int b = 4 * C + t;
              if (a < NN && b < NN && a <= b && (ii == 0 || a < b)) {
                const double kxx = c11 * mxx + mu * myy;
                const double kxy = lam * mxy + mu * myx;
                const double kyx = lam * myx + mu * mxy;
                const double kyy = c11 * myy + mu * mxx;
                // the ring slot's previous bulk read (NSLOT writes ago) is complete
                asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(L::NSLOT - 1) : "memory");
                double *slot = reds + 128 * (nw % L::NSLOT);
                nw++;
                if constexpr (PLAN) {
                  frag_write<P>(O, el, a, b, ii, kxx, kxy, kyx, kyy, slot);
                } else {
                  frag_add_mapped<P>(O, el, a, b, ii, kxx, kxy, kyx, kyy, slot);
                }
              }
            }
          }
        };
        if constexpr (JAC) {
          static_assert(K4 == 7, "tile-pair groups of the order-4 layout");
          // compiler barriers keep each group's table loads inside the group (hoisting
          // them across groups raises register pressure past the budget)
          asm volatile("" ::: "memory");
          group(IC<0>{}, IC<3>{}, IC<0>{}, IC<3>{}, std::true_type{});
          asm volatile("" ::: "memory");
          group(IC<0>{}, IC<3>{}, IC<3>{}, IC<5>{}, std::true_type{});
          asm volatile("" ::: "memory");
          group(IC<0>{}, IC<3>{}, IC<5>{}, IC<7>{}, std::true_type{});
          if constexpr (RES) res_write();
          asm volatile("" ::: "memory");
          group(IC<3>{}, IC<5>{}, IC<3>{}, IC<7>{}, std::false_type{});
          asm volatile("" ::: "memory");
          group(IC<5>{}, IC<7>{}, IC<5>{}, IC<7>{}, std::false_type{});
        }
      }
    }
    if constexpr (Gen::kSched) {
      if (cur.last) gen.release(cur, lane);
    }
    __syncwarp();
    cur = nxt;
    nxt = nn2;
  }
  cp_async_wait_all();
  // bulk reductions complete (shared-memory reads and global writes) before exit
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// One mesh: plan mode, list positions [A.begin, A.begin + A.count) of one colour;
// drop-in mode, elements [A.begin, A.begin + A.count) through the reference map.
template <int P, int MODE>
__global__ void __launch_bounds__(32 * FragDims<P>::WARPS, FEM_FRAG_MINB) frag_kernel(const __grid_constant__ AsmArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  frag_prologue<P, (MODE & kB16) != 0>(smem);
  const int warp = threadIdx.x >> 5;
  PairStride gen{A.begin, A.begin + A.count, (int64_t)blockIdx.x * FragDims<P>::WARPS + warp,
                 (int64_t)gridDim.x * FragDims<P>::WARPS};
  frag_loop<P, MODE>(smem, gen, A, &A);
}

// One mesh, several list-position ranges (plan mode).
template <int P, int MODE>
__global__ void __launch_bounds__(32 * FragDims<P>::WARPS, FEM_FRAG_MINB)
    frag_ranges_kernel(const __grid_constant__ AsmArgs A, const RangeList R) {
  extern __shared__ __align__(16) unsigned char smem[];
  frag_prologue<P, (MODE & kB16) != 0>(smem);
  const int warp = threadIdx.x >> 5;
  PairRanges gen{R, (int64_t)blockIdx.x * FragDims<P>::WARPS + warp, (int64_t)gridDim.x * FragDims<P>::WARPS};
  frag_loop<P, MODE>(smem, gen, A, &A);
}

// One mesh, all colours in one dependency-ordered persistent launch (plan mode).
template <int P, int MODE>
__global__ void __launch_bounds__(32 * FragDims<P>::WARPS, FEM_FRAG_MINB)
    frag_sched_kernel(const __grid_constant__ AsmArgs A, const __grid_constant__ SchedArgs S) {
  extern __shared__ __align__(16) unsigned char smem[];
  frag_prologue<P, (MODE & kB16) != 0>(smem);
  PairSched gen{&S};
  frag_loop<P, MODE>(smem, gen, A, &A);
}

// Many meshes of one order, all colours in one dependency-ordered persistent launch:
// the tiles of every (mesh, colour) group, colours outermost, each group waiting
// for its mesh's previous colour.
template <int P, int MODE>
__global__ void __launch_bounds__(32 * FragDims<P>::WARPS, FEM_FRAG_MINB)
    frag_batched_sched_kernel(const AsmArgs *__restrict__ meshes, const __grid_constant__ SchedArgs S) {
  extern __shared__ __align__(16) unsigned char smem[];
  frag_prologue<P, (MODE & kB16) != 0>(smem);
  PairSchedT<true> gen{&S};
  frag_loop<P, MODE>(smem, gen, meshes[0], meshes);
}

// Many meshes of one order (one colour each): warps pull tiles from the launch's queue.
template <int P, int MODE>
__global__ void __launch_bounds__(32 * FragDims<P>::WARPS, FEM_FRAG_MINB)
    frag_batched_kernel(const AsmArgs *__restrict__ meshes, const Tile *__restrict__ tiles, int ntiles, int *counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  frag_prologue<P, (MODE & kB16) != 0>(smem);
  PairQueue gen{tiles, ntiles, counter, 0, 0, 0, false};
  frag_loop<P, MODE>(smem, gen, meshes[0], meshes);
}

// A launch whose grid may begin while the kernel before it on the stream drains
// (programmatic dependent launch): consecutive colour or band launches of one
// assembly overlap one's tail with the next one's table setup, gathers and element
// arithmetic; the fragment kernel waits for the previous grid before it writes.
template <typename K, typename... Args>
cudaError_t pdl_launch(K kernel, int grid, int nt, size_t smem, cudaStream_t s, const Args &...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)nt);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// chained: the launch follows this assembly's previous fragment-kernel launch on the
// stream (a later colour or band), whose outputs are the only ones it may read
// early, so it may start as that one drains; a first launch follows the caller's
// work, which may have produced its inputs, and launches in stream order.
template <int P, int MODE>
int launch_frag_p(const AsmArgs &a, cudaStream_t s, bool chained) {
  using F = FragDims<P>;
  constexpr int NT = 32 * F::WARPS;
  auto kernel = frag_kernel<P, MODE>;
  const size_t smem = FragLayout<P, (MODE & kPlan) == 0, (MODE & kNL) != 0, (MODE & kB16) != 0, (MODE & kJac) != 0>::total;
  LaunchInfo li;
  int st = launch_info(kernel, NT, smem, li);
  if (st) return st;
  const int64_t pairs = (a.count + 1) / 2;
  const int64_t need = (pairs + F::WARPS - 1) / F::WARPS;
  // Order-3 drop-in Jacobian (every block added through the element map, one launch
  // whose elements share blocks): two CTAs per SM.  At 1024^2 the kernel took 3.90 ms
  // with two resident CTAs per SM against 4.35 ms with three (the bulk reductions of
  // more warps contend in L2); at order 2 (four CTAs) halving them cost 2.04 -> 3.46
  // ms on the 512x2048 annulus, so it keeps its occupancy.
  const int perSm =
      (P == 3 && (MODE & kPlan) == 0 && (MODE & kJac) != 0) ? std::min(li.grid_per_sm, 2) : li.grid_per_sm;
  const int64_t cap = (int64_t)perSm * li.num_sms;
  const int grid = (int)(need < cap ? need : cap);
  if (grid <= 0) return FEM_SUCCESS;
  cudaError_t err;
  if (chained) {
    err = pdl_launch(kernel, grid, NT, smem, s, a);
  } else {
    kernel<<<grid, NT, smem, s>>>(a);
    err = cudaGetLastError();
  }
  if (err != cudaSuccess) return cuda_fail(err, "frag_kernel launch");
  return FEM_SUCCESS;
}

template <int P, int MODE>
int launch_frag_ranges_p(const AsmArgs &a, const RangeList &r, cudaStream_t s, bool chained) {
  using F = FragDims<P>;
  constexpr int NT = 32 * F::WARPS;
  auto kernel = frag_ranges_kernel<P, MODE>;
  const size_t smem = FragLayout<P, false, (MODE & kNL) != 0, (MODE & kB16) != 0, (MODE & kJac) != 0>::total;
  LaunchInfo li;
  int st = launch_info(kernel, NT, smem, li);
  if (st) return st;
  int64_t pairs = 0;
  for (int i = 0; i < r.n; i++) pairs += (r.count[i] + 1) / 2;
  const int64_t need = (pairs + F::WARPS - 1) / F::WARPS;
  const int64_t cap = (int64_t)li.grid_per_sm * li.num_sms;
  const int grid = (int)(need < cap ? need : cap);
  if (grid <= 0) return FEM_SUCCESS;
  cudaError_t err;
  if (chained) {
    err = pdl_launch(kernel, grid, NT, smem, s, a, r);
  } else {
    kernel<<<grid, NT, smem, s>>>(a, r);
    err = cudaGetLastError();
  }
  if (err != cudaSuccess) return cuda_fail(err, "frag_ranges_kernel launch");
  return FEM_SUCCESS;
}

template <int P, int MODE>
int launch_frag_batched_p(const AsmArgs *meshes, const Tile *tiles, int ntiles, int *counter, cudaStream_t s) {
  using F = FragDims<P>;
  constexpr int NT = 32 * F::WARPS;
  auto kernel = frag_batched_kernel<P, MODE>;
  const size_t smem = FragLayout<P, false, false, (MODE & kB16) != 0>::total;
  LaunchInfo li;
  int st = launch_info(kernel, NT, smem, li);
  if (st) return st;
  const int64_t need = (ntiles + F::WARPS - 1) / F::WARPS;
  const int64_t cap = (int64_t)li.grid_per_sm * li.num_sms;
  const int grid = (int)(need < cap ? need : cap);
  if (grid <= 0) return FEM_SUCCESS;
  kernel<<<grid, NT, smem, s>>>(meshes, tiles, ntiles, counter);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "frag_batched_kernel launch");
  return FEM_SUCCESS;
}

template <int P, int MODE>
int launch_frag_batched_sched_p(const AsmArgs *meshes, const SchedArgs &sa, cudaStream_t s) {
  using F = FragDims<P>;
  constexpr int NT = 32 * F::WARPS;
  auto kernel = frag_batched_sched_kernel<P, MODE>;
  const size_t smem = FragLayout<P, false, false, (MODE & kB16) != 0>::total;
  LaunchInfo li;
  int st = launch_info(kernel, NT, smem, li);
  if (st) return st;
  const int64_t need = ((int64_t)sa.ntiles + F::WARPS - 1) / F::WARPS;
  const int64_t cap = (int64_t)li.grid_per_sm * li.num_sms;
  const int grid = (int)(need < cap ? need : cap);
  if (grid <= 0) return FEM_SUCCESS;
  kernel<<<grid, NT, smem, s>>>(meshes, sa);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "frag_batched_sched_kernel launch");
  return FEM_SUCCESS;
}

template <int P, int MODE>
int launch_frag_sched_p(const AsmArgs &a, const SchedArgs &sa, cudaStream_t s) {
  using F = FragDims<P>;
  constexpr int NT = 32 * F::WARPS;
  auto kernel = frag_sched_kernel<P, MODE>;
  const size_t smem = FragLayout<P, false, (MODE & kNL) != 0, (MODE & kB16) != 0, (MODE & kJac) != 0>::total;
  LaunchInfo li;
  int st = launch_info(kernel, NT, smem, li);
  if (st) return st;
  const int64_t need = ((int64_t)sa.ntiles + F::WARPS - 1) / F::WARPS;
  const int64_t cap = (int64_t)li.grid_per_sm * li.num_sms;
  const int grid = (int)(need < cap ? need : cap);
  if (grid <= 0) return FEM_SUCCESS;
  kernel<<<grid, NT, smem, s>>>(a, sa);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "frag_sched_kernel launch");
  return FEM_SUCCESS;
}

template <int MODE>
int launch_frag_mode(int order, const AsmArgs &a, cudaStream_t s, bool chained) {
  switch (order) {
    case 2:
      if constexpr ((MODE & kB16) != 0) return fail(FEM_ERR_INVALID_ORDER, "fragment kernel, BF16x6: order 2");
      else return launch_frag_p<2, MODE>(a, s, chained);
    case 3: return launch_frag_p<3, MODE>(a, s, chained);
    case 4:
      if constexpr ((MODE & (kNL | kB16)) != 0) return fail(FEM_ERR_INVALID_ORDER, "fragment kernel, mode %d: order 4", MODE);
      else return launch_frag_p<4, MODE>(a, s, chained);
    default: return fail(FEM_ERR_INVALID_ORDER, "fragment kernel: order %d", order);
  }
}

}  // namespace dev

// MIXED, LINEAR, order 3: the Jacobian's element stiffness runs as BF16x6 tensor-core
// products (kB16); everything else of the kernel stays FP64.  Order 2 pads 9 nodes and
// 9 quadrature points to 16 in both operands and ran slower than FP64 (2.0 against
// 1.4 ms on the 512x2048 annulus), so MIXED keeps the FP64 kernel there.
bool b16_stiffness(int order, int precision, int strain) {
  return precision == FEM_PRECISION_MIXED && strain == FEM_STRAIN_LINEAR && order == 3;
}

// FP64, LINEAR: orders 2 and 3 in every mode; order 4 in plan mode only (single
// meshes, batches, the server): measured on B200, the order-4 fragment kernel runs
// the 256-mesh batch in 170 against 217 ms and one 512^2 mesh in 3.03 against
// 3.00 ms for the element kernel, and plans and batches must run the same kernel
// (a mesh's batched result equals its single-mesh plan result bit for bit); the
// order-4 drop-in keeps the element kernel (4.7 ms against 6.9 ms).
// MIXED at orders 2 and 3 also runs this kernel (faster than the FP32 element
// products there: 3.1 against 3.8 ms at 1024^2 p = 3): at order 3 with the element
// stiffness as BF16x6 tensor-core products (b16_stiffness), at order 2 in FP64 (the
// FP64 result, as order-1 row assembly gives); at order 4 the FP32 element kernel is
// the faster one (2.6 against 3.4 ms) and MIXED keeps it.
bool frag_supported(int order, int precision, int strain, bool plan) {
  if (strain == FEM_STRAIN_NONLINEAR) return precision == FEM_PRECISION_FP64 && (order == 2 || order == 3);
  if (strain != FEM_STRAIN_LINEAR) return false;
  if (precision == FEM_PRECISION_MIXED) return order == 2 || order == 3;
  if (precision != FEM_PRECISION_FP64) return false;
  return order == 2 || order == 3 || (order == 4 && plan);
}

int launch_frag(int order, int precision, int mode, const dev::AsmArgs &a, cudaStream_t s, int strain, bool chained) {
  using namespace dev;
  if (strain == FEM_STRAIN_NONLINEAR) mode |= kNL;
  if (b16_stiffness(order, precision, strain) && (mode & kJac)) mode |= kB16;
  switch (mode) {
    case kPlan | kJac | kB16: return launch_frag_mode<kPlan | kJac | kB16>(order, a, s, chained);
    case kPlan | kRes | kJac | kB16: return launch_frag_mode<kPlan | kRes | kJac | kB16>(order, a, s, chained);
    case kJac | kB16: return launch_frag_mode<kJac | kB16>(order, a, s, chained);
    case kRes | kJac | kB16: return launch_frag_mode<kRes | kJac | kB16>(order, a, s, chained);
    case kPlan | kRes: return launch_frag_mode<kPlan | kRes>(order, a, s, chained);
    case kPlan | kJac: return launch_frag_mode<kPlan | kJac>(order, a, s, chained);
    case kPlan | kRes | kJac: return launch_frag_mode<kPlan | kRes | kJac>(order, a, s, chained);
    case kRes: return launch_frag_mode<kRes>(order, a, s, chained);
    case kJac: return launch_frag_mode<kJac>(order, a, s, chained);
    case kRes | kJac: return launch_frag_mode<kRes | kJac>(order, a, s, chained);
    case kNL | kPlan | kRes: return launch_frag_mode<kNL | kPlan | kRes>(order, a, s, chained);
    case kNL | kPlan | kJac: return launch_frag_mode<kNL | kPlan | kJac>(order, a, s, chained);
    case kNL | kPlan | kRes | kJac: return launch_frag_mode<kNL | kPlan | kRes | kJac>(order, a, s, chained);
    case kNL | kRes: return launch_frag_mode<kNL | kRes>(order, a, s, chained);
    case kNL | kJac: return launch_frag_mode<kNL | kJac>(order, a, s, chained);
    case kNL | kRes | kJac: return launch_frag_mode<kNL | kRes | kJac>(order, a, s, chained);
    default: return fail(FEM_ERR_INVALID_ARGUMENT, "fragment kernel: mode %d", mode);
  }
}

int launch_frag_ranges(int order, int precision, int mode, const dev::AsmArgs &a, const dev::RangeList &r,
                       cudaStream_t s, int strain, bool chained) {
  using namespace dev;
  if (strain == FEM_STRAIN_NONLINEAR) mode |= kNL;
  if (b16_stiffness(order, precision, strain) && (mode & kJac)) mode |= kB16;
  auto go = [&](auto mc) -> int {
    constexpr int M = decltype(mc)::value;
    switch (order) {
      case 2:
        if constexpr ((M & kB16) != 0) return fail(FEM_ERR_INVALID_ORDER, "fragment kernel, BF16x6: order 2");
        else return launch_frag_ranges_p<2, M>(a, r, s, chained);
      case 3: return launch_frag_ranges_p<3, M>(a, r, s, chained);
      case 4:
        if constexpr ((M & (kNL | kB16)) != 0) return fail(FEM_ERR_INVALID_ORDER, "fragment kernel, mode %d: order 4", M);
        else return launch_frag_ranges_p<4, M>(a, r, s, chained);
      default: return fail(FEM_ERR_INVALID_ORDER, "fragment kernel: order %d", order);
    }
  };
  switch (mode) {
    case kPlan | kRes: return go(IC<kPlan | kRes>{});
    case kPlan | kRes | kJac: return go(IC<kPlan | kRes | kJac>{});
    case kPlan | kRes | kJac | kB16: return go(IC<kPlan | kRes | kJac | kB16>{});
    case kNL | kPlan | kRes: return go(IC<kNL | kPlan | kRes>{});
    case kNL | kPlan | kRes | kJac: return go(IC<kNL | kPlan | kRes | kJac>{});
    default: return fail(FEM_ERR_INVALID_ARGUMENT, "fragment kernel, ranges: mode %d", mode);
  }
}

int launch_frag_sched(int order, int precision, int mode, const dev::AsmArgs &a, const dev::SchedArgs &sa,
                      cudaStream_t s, int strain) {
  using namespace dev;
  if (strain == FEM_STRAIN_NONLINEAR) mode |= kNL;
  if (b16_stiffness(order, precision, strain) && (mode & kJac)) mode |= kB16;
  auto go = [&](auto mc) -> int {
    constexpr int M = decltype(mc)::value;
    switch (order) {
      case 2:
        if constexpr ((M & kB16) != 0) return fail(FEM_ERR_INVALID_ORDER, "fragment kernel, BF16x6: order 2");
        else return launch_frag_sched_p<2, M>(a, sa, s);
      case 3: return launch_frag_sched_p<3, M>(a, sa, s);
      case 4:
        if constexpr ((M & (kNL | kB16)) != 0) return fail(FEM_ERR_INVALID_ORDER, "fragment kernel, mode %d: order 4", M);
        else return launch_frag_sched_p<4, M>(a, sa, s);
      default: return fail(FEM_ERR_INVALID_ORDER, "fragment kernel: order %d", order);
    }
  };
  switch (mode) {
    case kPlan | kRes: return go(IC<kPlan | kRes>{});
    case kPlan | kJac: return go(IC<kPlan | kJac>{});
    case kPlan | kRes | kJac: return go(IC<kPlan | kRes | kJac>{});
    case kPlan | kJac | kB16: return go(IC<kPlan | kJac | kB16>{});
    case kPlan | kRes | kJac | kB16: return go(IC<kPlan | kRes | kJac | kB16>{});
    case kNL | kPlan | kRes: return go(IC<kNL | kPlan | kRes>{});
    case kNL | kPlan | kJac: return go(IC<kNL | kPlan | kJac>{});
    case kNL | kPlan | kRes | kJac: return go(IC<kNL | kPlan | kRes | kJac>{});
    default: return fail(FEM_ERR_INVALID_ARGUMENT, "fragment kernel, schedule: mode %d", mode);
  }
}

int launch_frag_batched_sched(int order, int precision, const dev::AsmArgs *meshes, const dev::SchedArgs &sa,
                              cudaStream_t s) {
  using namespace dev;
  constexpr int M = kPlan | kRes | kJac;
  const bool b16 = b16_stiffness(order, precision, FEM_STRAIN_LINEAR);
  switch (order) {
    case 2: return launch_frag_batched_sched_p<2, M>(meshes, sa, s);
    case 3: return b16 ? launch_frag_batched_sched_p<3, M | kB16>(meshes, sa, s)
                       : launch_frag_batched_sched_p<3, M>(meshes, sa, s);
    case 4: return launch_frag_batched_sched_p<4, M>(meshes, sa, s);
    default: return fail(FEM_ERR_INVALID_ORDER, "fragment kernel: order %d", order);
  }
}

int launch_frag_batched(int order, int precision, const dev::AsmArgs *meshes, const dev::Tile *tiles, int ntiles,
                        int *counter, cudaStream_t s) {
  using namespace dev;
  constexpr int M = kPlan | kRes | kJac;
  const bool b16 = b16_stiffness(order, precision, FEM_STRAIN_LINEAR);
  switch (order) {
    case 2: return launch_frag_batched_p<2, M>(meshes, tiles, ntiles, counter, s);
    case 3: return b16 ? launch_frag_batched_p<3, M | kB16>(meshes, tiles, ntiles, counter, s)
                       : launch_frag_batched_p<3, M>(meshes, tiles, ntiles, counter, s);
    case 4: return launch_frag_batched_p<4, M>(meshes, tiles, ntiles, counter, s);
    default: return fail(FEM_ERR_INVALID_ORDER, "fragment kernel: order %d", order);
  }
}

}  // namespace fem
