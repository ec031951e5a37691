// Row assembly of order-1 meshes: every BSR block row is written exactly once.
//
// The element kernels scatter an element's 2x2 blocks to the rows of its nodes;
// at p = 1 a vertex row is shared by four elements, so 7 of an element's 16
// blocks are later-colour reductions (4 scalar RED.f64 each) and every block is
// a scattered 32-byte store.  Here a warp owns a chunk of up to 32 consecutive
// rows (kRowChunkRows, at most kRowChunkBlocks blocks) and lane l owns row
// r0 + l: it walks the elements listing r (the plan's rowElem table, in colour
// order), recomputes each element's quadrature data (J, J^-1, the gradients,
// the weak stress; 4 points) and adds the element's row slice
//   K[(a,i),(b,k)] = lam M_ik + mu M_ki + mu delta_ik (M_xx + M_yy),
//   M_ij = sum_q s G_ai G_bj,  R_ai = sum_q s (sigma G_a)_i
// (the closed form of the reference's forward-mode column, element/FEKernels.h:
// 286-315,884-976) into the chunk's blocks in shared memory.  The warp then
// streams the chunk's blocks [rowp[r0], rowp[r1]) to HBM with consecutive
// 32-byte stores (each instruction 1 KB contiguous) and the residual rows with
// consecutive 16-byte stores: no zeroing, no atomics, one launch, deterministic
// (each row sums its elements in colour order).  The price is that each element's
// quadrature stage runs once per node row (4x at p = 1); the arithmetic stays in
// FP64 for both precisions.
#include <cuda_runtime.h>

#include <cstdint>

#include "fem_common.h"
#include "fem_device.cuh"
#include "fem_launch.h"

namespace fem {
namespace dev {

constexpr int kRowWarps = 4;

// Shared-memory position (in double2 units) of chunk block i: blocks are 32 bytes
// apart with 16 more bytes after every 9 (the row length of a structured p = 1
// mesh), so the 32 lanes' rows start in different banks; a function of i alone,
// so the streaming store needs no row lookup.
__device__ __forceinline__ int acc_pos(int i) { return 2 * i + i / 9; }
constexpr int kAccUnits = 2 * kRowChunkBlocks + kRowChunkBlocks / 9 + 1;  // double2 per warp

// A chunk's header as one lane sees it: the chunk's rows [r0, r1) and blocks
// [blk0, blk0 + nb), the lane's row r0 + lane, its first block relative to blk0
// and its rowElem entries [j0, j1) (empty past r1).
struct RowHead {
  int r0, r1, blk0, nb, base, j0, j1;
};

__device__ __forceinline__ RowHead row_head(const AsmArgs &M, int r0, int r1, int lane) {
  RowHead h{r0, r1, 0, 0, 0, 0, 0};
  h.blk0 = __ldg(M.rowp + r0);
  h.nb = __ldg(M.rowp + r1) - h.blk0;
  const int r = r0 + lane;
  if (r < r1) {
    h.base = __ldg(M.rowp + r) - h.blk0;
    h.j0 = __ldg(M.rowElemPtr + r);
    h.j1 = __ldg(M.rowElemPtr + r + 1);
  }
  return h;
}

// Chunks c, c + stride, ... < end of mesh M, by the calling warp; acc is the
// warp's kAccUnits double2 of shared memory.  NP, NM: the 1D basis values at the
// Gauss point on the node's own side / the opposite side, fma(0.5, g, 0.5) and
// fma(-0.5, g, 0.5) as in lagrangePoly1dDeriv<double,1>.  For the bilinear
// element the xi-column of J = sum_b x_b (x) dN_b depends on the point's eta only
// and the eta-column on its xi only: with the edge vectors e0 = x1 - x0,
// e1 = x3 - x2, f0 = x2 - x0, f1 = x3 - x1, dx/dxi(qy) = (NP e_qy + NM e_(1-qy)) / 2
// and dx/deta(qx) = (NP f_qx + NM f_(1-qx)) / 2 (likewise for the states).
//
// The loads run ahead of the arithmetic across chunk boundaries, so that a chunk
// does not start with its dependent chain (row range -> row pointers and element
// ranges -> rowElem entry -> node ids -> coordinates and states) exposed: the row
// range of the chunk after next and the header of the next chunk are loaded when a
// chunk starts, and each lane's element pipeline (nodal data one entry ahead,
// rowElem entry and node ids two ahead) runs over the lane's entries of the
// current chunk followed by those of the next.
template <int MODE>
__device__ __forceinline__ void row_stream(const AsmArgs &M, int64_t c, int64_t end, int64_t stride, double2 *acc,
                                           int lane, double NP, double NM) {
  if (c >= end) return;
  const double mu = M.mu, lam = M.lam, thick = M.t, c11 = lam + 2.0 * mu;
  const double hP = 0.5 * NP, hM = 0.5 * NM;
  const int2 *rowElem = reinterpret_cast<const int2 *>(M.rowElem);
  const int4 *conn4 = reinterpret_cast<const int4 *>(M.connList);
  const double2 *X2 = reinterpret_cast<const double2 *>(M.coords);
  const double2 *U2 = reinterpret_cast<const double2 *>(M.states);
  RowHead h = row_head(M, __ldg(M.rowChunk + c), __ldg(M.rowChunk + c + 1), lane);
  int64_t cn = c + stride;
  int n0 = 0, n1 = 0;  // row range of chunk cn
  if (cn < end) n0 = __ldg(M.rowChunk + cn), n1 = __ldg(M.rowChunk + cn + 1);
  // element pipeline over this lane's entries (current chunk, then next chunk):
  // nodal data of entry k in x/u and its rowElem entry in enC, entry k + 1 in enN/ndN
  int2 enC = make_int2(0, 0), enN = make_int2(0, 0);
  int4 ndN = make_int4(0, 0, 0, 0);
  double2 x[4], u[4];
  auto load_nodes = [&](int4 nd) {
    x[0] = __ldg(X2 + nd.x), x[1] = __ldg(X2 + nd.y), x[2] = __ldg(X2 + nd.z), x[3] = __ldg(X2 + nd.w);
    u[0] = __ldg(U2 + nd.x), u[1] = __ldg(U2 + nd.y), u[2] = __ldg(U2 + nd.z), u[3] = __ldg(U2 + nd.w);
  };
  int lenC = h.j1 - h.j0;
  if (lenC > 0) {
    enC = __ldg(rowElem + h.j0);
    load_nodes(__ldg(conn4 + (enC.x >> 2)));
  }
  if (lenC > 1) {
    enN = __ldg(rowElem + h.j0 + 1);
    ndN = __ldg(conn4 + (enN.x >> 2));
  }
  for (;;) {
    const bool hasN = cn < end;
    RowHead hn{0, 0, 0, 0, 0, 0, 0};
    if (hasN) hn = row_head(M, n0, n1, lane);
    const int64_t cnn = cn + stride;
    if (hasN && cnn < end) n0 = __ldg(M.rowChunk + cnn), n1 = __ldg(M.rowChunk + cnn + 1);
    const int lenN = hn.j1 - hn.j0, tot = lenC + lenN;
    if (lenC == 1 && lenN > 0) {  // entry 1 is the next chunk's first
      enN = __ldg(rowElem + hn.j0);
      ndN = __ldg(conn4 + (enN.x >> 2));
    }
    if constexpr ((MODE & kJac) != 0) {
      for (int i = lane; i < h.nb; i += 32) {
        acc[acc_pos(i)] = make_double2(0.0, 0.0);
        acc[acc_pos(i) + 1] = make_double2(0.0, 0.0);
      }
    }
    __syncwarp();
    double rx = 0.0, ry = 0.0;
    for (int k = 0; k < lenC; k++) {
      // J and grad-u columns at the two eta (xi-derivative) and two xi (eta-derivative) values
      double2 Jxi[2], Jeta[2], Uxi[2], Ueta[2];
      {
        const double2 e0 = make_double2(x[1].x - x[0].x, x[1].y - x[0].y);
        const double2 e1 = make_double2(x[3].x - x[2].x, x[3].y - x[2].y);
        const double2 f0 = make_double2(x[2].x - x[0].x, x[2].y - x[0].y);
        const double2 f1 = make_double2(x[3].x - x[1].x, x[3].y - x[1].y);
        const double2 a0 = make_double2(u[1].x - u[0].x, u[1].y - u[0].y);
        const double2 a1 = make_double2(u[3].x - u[2].x, u[3].y - u[2].y);
        const double2 b0 = make_double2(u[2].x - u[0].x, u[2].y - u[0].y);
        const double2 b1 = make_double2(u[3].x - u[1].x, u[3].y - u[1].y);
        Jxi[0] = make_double2(hP * e0.x + hM * e1.x, hP * e0.y + hM * e1.y);
        Jxi[1] = make_double2(hM * e0.x + hP * e1.x, hM * e0.y + hP * e1.y);
        Jeta[0] = make_double2(hP * f0.x + hM * f1.x, hP * f0.y + hM * f1.y);
        Jeta[1] = make_double2(hM * f0.x + hP * f1.x, hM * f0.y + hP * f1.y);
        Uxi[0] = make_double2(hP * a0.x + hM * a1.x, hP * a0.y + hM * a1.y);
        Uxi[1] = make_double2(hM * a0.x + hP * a1.x, hM * a0.y + hP * a1.y);
        Ueta[0] = make_double2(hP * b0.x + hM * b1.x, hP * b0.y + hM * b1.y);
        Ueta[1] = make_double2(hM * b0.x + hP * b1.x, hM * b0.y + hP * b1.y);
      }
      const int2 en = enC;
      // prefetch: nodal data of entry k + 1, rowElem entry and node ids of entry k + 2
      if (k + 1 < tot) {
        load_nodes(ndN);
        enC = enN;
      }
      if (k + 2 < tot) {
        enN = __ldg(rowElem + (k + 2 < lenC ? h.j0 + k + 2 : hn.j0 + (k + 2 - lenC)));
        ndN = __ldg(conn4 + (enN.x >> 2));
      }
      const int a = en.x & 3, ax = a & 1, ay = a >> 1;
      double Mm[4][4];  // sum_q s G_ai G_bj per column node b: [b][xx, xy, yx, yy]
#pragma unroll
      for (int b = 0; b < 4; b++) Mm[b][0] = Mm[b][1] = Mm[b][2] = Mm[b][3] = 0.0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int qx = q & 1, qy = q >> 1;
        const double j00 = Jxi[qy].x, j10 = Jxi[qy].y, j01 = Jeta[qx].x, j11 = Jeta[qx].y;
        const double g00 = Uxi[qy].x, g10 = Uxi[qy].y, g01 = Ueta[qx].x, g11 = Ueta[qx].y;
        const double det = j00 * j11 - j01 * j10;
        const double inv = 1.0 / det;
        const double i00 = j11 * inv, i01 = -j01 * inv, i10 = -j10 * inv, i11 = j00 * inv;
        const double st = det * thick;  // the 2x2 Gauss weights are 1
        const double uxx = g00 * i00 + g01 * i10, uxy = g00 * i01 + g01 * i11;
        const double uyx = g10 * i00 + g11 * i10, uyy = g10 * i01 + g11 * i11;
        const double tr = uxx + uyy;
        const double sxx = 2.0 * mu * uxx + lam * tr, sxy = mu * (uxy + uyx), syy = 2.0 * mu * uyy + lam * tr;
        double gx[4], gy[4];
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const int bx = b & 1, by = b >> 1;
          const double dxi = (by == qy ? hP : hM) * (bx ? 1.0 : -1.0);
          const double deta = (bx == qx ? hP : hM) * (by ? 1.0 : -1.0);
          gx[b] = dxi * i00 + deta * i10;
          gy[b] = dxi * i01 + deta * i11;
        }
        // the row node's own gradient, from its tabulated derivatives
        const double dxa = (ay == qy ? hP : hM) * (ax ? 1.0 : -1.0);
        const double dea = (ax == qx ? hP : hM) * (ay ? 1.0 : -1.0);
        const double hx = st * (dxa * i00 + dea * i10), hy = st * (dxa * i01 + dea * i11);
        rx = fma(hx, sxx, fma(hy, sxy, rx));
        ry = fma(hx, sxy, fma(hy, syy, ry));
#pragma unroll
        for (int b = 0; b < 4; b++) {
          Mm[b][0] = fma(hx, gx[b], Mm[b][0]);
          Mm[b][1] = fma(hx, gy[b], Mm[b][1]);
          Mm[b][2] = fma(hy, gx[b], Mm[b][2]);
          Mm[b][3] = fma(hy, gy[b], Mm[b][3]);
        }
      }
      if constexpr ((MODE & kJac) != 0) {
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const double kxx = c11 * Mm[b][0] + mu * Mm[b][3];
          const double kxy = lam * Mm[b][1] + mu * Mm[b][2];
          const double kyx = lam * Mm[b][2] + mu * Mm[b][1];
          const double kyy = c11 * Mm[b][3] + mu * Mm[b][0];
          double2 *sp = acc + acc_pos(h.base + ((en.y >> (8 * b)) & 0xff));
          const double2 p0 = sp[0], p1 = sp[1];
          sp[0] = make_double2(p0.x + kxx, p0.y + kxy);
          sp[1] = make_double2(p1.x + kyx, p1.y + kyy);
        }
      }
    }
    __syncwarp();
    if constexpr ((MODE & kRes) != 0) {
      if (h.r0 + lane < h.r1) reinterpret_cast<double2 *>(M.residual)[h.r0 + lane] = make_double2(rx, ry);
    }
    if constexpr ((MODE & kJac) != 0) {
      double *dst = M.mat + 4 * (int64_t)h.blk0;
      for (int i = lane; i < h.nb; i += 32) {
        const double2 p0 = acc[acc_pos(i)], p1 = acc[acc_pos(i) + 1];
        store_block(dst + 4 * i, p0.x, p0.y, p1.x, p1.y);
      }
    }
    __syncwarp();
    if (!hasN) break;
    if (lenC == 0 && lenN > 0) {  // this lane's pipeline starts in the next chunk
      enC = __ldg(rowElem + hn.j0);
      load_nodes(__ldg(conn4 + (enC.x >> 2)));
      if (lenN > 1) {
        enN = __ldg(rowElem + hn.j0 + 1);
        ndN = __ldg(conn4 + (enN.x >> 2));
      }
    }
    h = hn;
    lenC = lenN;
    cn = cnn;
  }
}

__device__ __forceinline__ void p1_basis(double &NP, double &NM) {
  NP = __fma_rn(0.5, kGX[1][1], 0.5);
  NM = __fma_rn(-0.5, kGX[1][1], 0.5);
}

// Single mesh: chunks [A.begin, A.begin + A.count), grid-stride over warps.
template <int MODE>
__global__ void __launch_bounds__(32 * kRowWarps, 3) rows_p1_kernel(const __grid_constant__ AsmArgs A) {
  __shared__ double2 acc[kRowWarps][kAccUnits];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double NP, NM;
  p1_basis(NP, NM);
  row_stream<MODE>(A, A.begin + (int64_t)blockIdx.x * kRowWarps + warp, A.begin + A.count,
                   (int64_t)gridDim.x * kRowWarps, acc[warp], lane, NP, NM);
}

// Many meshes: warps pull tiles (mesh, `count` chunks from `begin`) from the queue.
__global__ void __launch_bounds__(32 * kRowWarps, 3) rows_p1_batched_kernel(const AsmArgs *__restrict__ meshes,
                                                                        const Tile *__restrict__ tiles, int ntiles,
                                                                        int *counter) {
  __shared__ double2 acc[kRowWarps][kAccUnits];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double NP, NM;
  p1_basis(NP, NM);
  int ahead = -1;  // lane 0: the next tile, taken one tile ahead (hides the queue atomic's latency)
  for (;;) {
    int t = 0;
    if (lane == 0) {
      t = ahead < 0 ? atomicAdd(counter, 1) : ahead;
      ahead = t < ntiles ? atomicAdd(counter, 1) : ntiles;
    }
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= ntiles) break;
    const Tile tl = tiles[t];
    const AsmArgs &M = meshes[tl.mesh];
    row_stream<kRes | kJac>(M, tl.begin, tl.begin + tl.count, 1, acc[warp], lane, NP, NM);
  }
}

}  // namespace dev

namespace {
template <typename K>
int grid_for(K kernel, int64_t work_warps, int &grid) {
  LaunchInfo li;
  int st = launch_info(kernel, 32 * dev::kRowWarps, 0, li);
  if (st) return st;
  const int64_t need = (work_warps + dev::kRowWarps - 1) / dev::kRowWarps;
  const int64_t cap = (int64_t)li.grid_per_sm * li.num_sms;
  grid = (int)(need < cap ? need : cap);
  return FEM_SUCCESS;
}
}  // namespace

int launch_rows(int mode, const dev::AsmArgs &a, cudaStream_t s) {
  using namespace dev;
  int grid = 0, st = FEM_SUCCESS;
  switch (mode & (kRes | kJac)) {
    case kRes:
      st = grid_for(rows_p1_kernel<kRes>, a.count, grid);
      if (!st && grid > 0) rows_p1_kernel<kRes><<<grid, 32 * kRowWarps, 0, s>>>(a);
      break;
    case kJac:
      st = grid_for(rows_p1_kernel<kJac>, a.count, grid);
      if (!st && grid > 0) rows_p1_kernel<kJac><<<grid, 32 * kRowWarps, 0, s>>>(a);
      break;
    case kRes | kJac:
      st = grid_for(rows_p1_kernel<kRes | kJac>, a.count, grid);
      if (!st && grid > 0) rows_p1_kernel<kRes | kJac><<<grid, 32 * kRowWarps, 0, s>>>(a);
      break;
    default: return fail(FEM_ERR_INVALID_ARGUMENT, "bad row-kernel mode %d", mode);
  }
  if (st) return st;
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "rows_p1_kernel launch");
  return FEM_SUCCESS;
}

int launch_rows_batched(const dev::AsmArgs *meshes, const dev::Tile *tiles, int ntiles, int *counter,
                        cudaStream_t s) {
  using namespace dev;
  int grid = 0;
  int st = grid_for(rows_p1_batched_kernel, (int64_t)ntiles, grid);
  if (st) return st;
  if (grid <= 0) return FEM_SUCCESS;
  rows_p1_batched_kernel<<<grid, 32 * kRowWarps, 0, s>>>(meshes, tiles, ntiles, counter);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "rows_p1_batched_kernel launch");
  return FEM_SUCCESS;
}

}  // namespace fem
