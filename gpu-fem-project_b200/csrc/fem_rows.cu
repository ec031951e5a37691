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

// One chunk c of mesh M, by the calling warp; acc is the warp's kRowChunkBlocks
// blocks of shared memory (two double2 per block).  NP, NM: the 1D basis values
// N(x) at the Gauss point on the node's own side / the opposite side,
// fma(0.5, g, 0.5) and fma(-0.5, g, 0.5) as in lagrangePoly1dDeriv<double,1>.
template <int MODE>
__device__ __forceinline__ void row_chunk(const AsmArgs &M, int64_t c, double2 *acc, int lane, double NP, double NM) {
  const int r0 = __ldg(M.rowChunk + c), r1 = __ldg(M.rowChunk + c + 1);
  const int blk0 = __ldg(M.rowp + r0), nb = __ldg(M.rowp + r1) - blk0;
  for (int i = lane; i < 2 * nb; i += 32) acc[i] = make_double2(0.0, 0.0);
  __syncwarp();
  const double mu = M.mu, lam = M.lam, thick = M.t, c11 = lam + 2.0 * mu;
  const int r = r0 + lane;
  double rx = 0.0, ry = 0.0;
  if (r < r1) {
    const int base = __ldg(M.rowp + r) - blk0;
    const int j1 = __ldg(M.rowElemPtr + r + 1);
    for (int j = __ldg(M.rowElemPtr + r); j < j1; j++) {
      const int2 en = __ldg(reinterpret_cast<const int2 *>(M.rowElem) + j);
      const int k = en.x >> 2, a = en.x & 3;
      const int4 nd = __ldg(reinterpret_cast<const int4 *>(M.connList) + k);
      const int node[4] = {nd.x, nd.y, nd.z, nd.w};
      double2 x[4], u[4];
#pragma unroll
      for (int b = 0; b < 4; b++) {
        x[b] = __ldg(reinterpret_cast<const double2 *>(M.coords) + node[b]);
        u[b] = __ldg(reinterpret_cast<const double2 *>(M.states) + node[b]);
      }
      double K[4][4];
#pragma unroll
      for (int b = 0; b < 4; b++) K[b][0] = K[b][1] = K[b][2] = K[b][3] = 0.0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int qx = q & 1, qy = q >> 1;
        // tabulated derivatives of node b = by*2+bx at point q = qy*2+qx (weights are 1)
        double dxi[4], deta[4];
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const int bx = b & 1, by = b >> 1;
          dxi[b] = (by == qy ? NP : NM) * (bx ? 0.5 : -0.5);
          deta[b] = (bx == qx ? NP : NM) * (by ? 0.5 : -0.5);
        }
        double j00 = 0, j01 = 0, j10 = 0, j11 = 0, g00 = 0, g01 = 0, g10 = 0, g11 = 0;
#pragma unroll
        for (int b = 0; b < 4; b++) {
          j00 = fma(x[b].x, dxi[b], j00);
          j01 = fma(x[b].x, deta[b], j01);
          j10 = fma(x[b].y, dxi[b], j10);
          j11 = fma(x[b].y, deta[b], j11);
          g00 = fma(u[b].x, dxi[b], g00);
          g01 = fma(u[b].x, deta[b], g01);
          g10 = fma(u[b].y, dxi[b], g10);
          g11 = fma(u[b].y, deta[b], g11);
        }
        const double det = j00 * j11 - j01 * j10;
        const double inv = 1.0 / det;
        const double i00 = j11 * inv, i01 = -j01 * inv, i10 = -j10 * inv, i11 = j00 * inv;
        const double st = det * thick;
        const double uxx = g00 * i00 + g01 * i10, uxy = g00 * i01 + g01 * i11;
        const double uyx = g10 * i00 + g11 * i10, uyy = g10 * i01 + g11 * i11;
        const double tr = uxx + uyy;
        const double sxx = 2.0 * mu * uxx + lam * tr, sxy = mu * (uxy + uyx), syy = 2.0 * mu * uyy + lam * tr;
        double gx[4], gy[4];
#pragma unroll
        for (int b = 0; b < 4; b++) {
          gx[b] = dxi[b] * i00 + deta[b] * i10;
          gy[b] = dxi[b] * i01 + deta[b] * i11;
        }
        const double gax = a == 0 ? gx[0] : a == 1 ? gx[1] : a == 2 ? gx[2] : gx[3];
        const double gay = a == 0 ? gy[0] : a == 1 ? gy[1] : a == 2 ? gy[2] : gy[3];
        const double hx = st * gax, hy = st * gay;
        rx = fma(hx, sxx, fma(hy, sxy, rx));
        ry = fma(hx, sxy, fma(hy, syy, ry));
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const double mxx = hx * gx[b], mxy = hx * gy[b], myx = hy * gx[b], myy = hy * gy[b];
          K[b][0] += c11 * mxx + mu * myy;
          K[b][1] += lam * mxy + mu * myx;
          K[b][2] += lam * myx + mu * mxy;
          K[b][3] += c11 * myy + mu * mxx;
        }
      }
      if constexpr ((MODE & kJac) != 0) {
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const int slot = base + ((en.y >> (8 * b)) & 0xff);
          double2 *s = acc + 2 * slot;
          const double2 p0 = s[0], p1 = s[1];
          s[0] = make_double2(p0.x + K[b][0], p0.y + K[b][1]);
          s[1] = make_double2(p1.x + K[b][2], p1.y + K[b][3]);
        }
      }
    }
  }
  __syncwarp();
  if constexpr ((MODE & kRes) != 0) {
    if (r < r1) reinterpret_cast<double2 *>(M.residual)[r] = make_double2(rx, ry);
  }
  if constexpr ((MODE & kJac) != 0) {
    double *dst = M.mat + 4 * (int64_t)blk0;
    for (int i = lane; i < nb; i += 32) {
      const double2 p0 = acc[2 * i], p1 = acc[2 * i + 1];
      store_block(dst + 4 * i, p0.x, p0.y, p1.x, p1.y);
    }
  }
  __syncwarp();
}

__device__ __forceinline__ void p1_basis(double &NP, double &NM) {
  NP = __fma_rn(0.5, kGX[1][1], 0.5);
  NM = __fma_rn(-0.5, kGX[1][1], 0.5);
}

// Single mesh: chunks [A.begin, A.begin + A.count), grid-stride over warps.
template <int MODE>
__global__ void __launch_bounds__(32 * kRowWarps) rows_p1_kernel(const __grid_constant__ AsmArgs A) {
  __shared__ double2 acc[kRowWarps][2 * kRowChunkBlocks];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double NP, NM;
  p1_basis(NP, NM);
  const int64_t end = A.begin + A.count, stride = (int64_t)gridDim.x * kRowWarps;
  for (int64_t c = A.begin + (int64_t)blockIdx.x * kRowWarps + warp; c < end; c += stride)
    row_chunk<MODE>(A, c, acc[warp], lane, NP, NM);
}

// Many meshes: warps pull tiles (mesh, `count` chunks from `begin`) from the queue.
__global__ void __launch_bounds__(32 * kRowWarps) rows_p1_batched_kernel(const AsmArgs *__restrict__ meshes,
                                                                        const Tile *__restrict__ tiles, int ntiles,
                                                                        int *counter) {
  __shared__ double2 acc[kRowWarps][2 * kRowChunkBlocks];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double NP, NM;
  p1_basis(NP, NM);
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(counter, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= ntiles) break;
    const Tile tl = tiles[t];
    const AsmArgs &M = meshes[tl.mesh];
    for (int64_t c = tl.begin; c < tl.begin + tl.count; c++) row_chunk<kRes | kJac>(M, c, acc[warp], lane, NP, NM);
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
