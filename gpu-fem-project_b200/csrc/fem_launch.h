// Host-side launch helpers shared by the single-mesh and batched entry points.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "fem_common.h"
#include "fem_device.cuh"

namespace fem {

struct LaunchInfo {
  int grid_per_sm = 0;
  int num_sms = 0;
};

inline std::mutex g_mu;
inline std::map<std::pair<const void *, int>, LaunchInfo> g_info;

inline int cuda_fail(cudaError_t err, const char *what) {
  return fail(FEM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(err));
}

// Occupancy-sized persistent grid; sets the dynamic shared-memory opt-in once per device.
template <typename K>
int launch_info(K kernel, int nt, size_t smem, LaunchInfo &out) {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return cuda_fail(err, "cudaGetDevice");
  std::lock_guard<std::mutex> lk(g_mu);
  auto key = std::make_pair(reinterpret_cast<const void *>(kernel), dev);
  auto it = g_info.find(key);
  if (it != g_info.end()) {
    out = it->second;
    return FEM_SUCCESS;
  }
  err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return cuda_fail(err, "cudaFuncSetAttribute");
  LaunchInfo li;
  err = cudaDeviceGetAttribute(&li.num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (err != cudaSuccess) return cuda_fail(err, "cudaDeviceGetAttribute");
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&li.grid_per_sm, kernel, nt, smem);
  if (err != cudaSuccess) return cuda_fail(err, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (li.grid_per_sm < 1) return fail(FEM_ERR_CUDA, "kernel does not fit on an SM (smem %zu B)", smem);
  g_info[key] = li;
  out = li;
  return FEM_SUCCESS;
}

// The occupancy query counts one CTA per SM for kernels that allocate tensor memory;
// the tcgen05 element kernel holds 64 of an SM's 512 TMEM columns per CTA, so its
// register and shared-memory limit (its minimum-blocks bound) is the real one.
template <int P, typename T, int MODE>
void umma_residency(LaunchInfo &li) {
  if constexpr ((MODE & dev::kU) != 0) li.grid_per_sm = std::max(li.grid_per_sm, dev::min_blocks<P, T, MODE>());
}

template <int P, typename T, int MODE>
int launch_p(const dev::AsmArgs &a, cudaStream_t s) {
  using S = dev::ShapeSel<P, MODE>;
  constexpr int NT = S::GT * S::GPC;
  auto kernel = dev::assemble_kernel<P, T, MODE>;
  const size_t smem = dev::Layout<P, T, MODE>::total;
  LaunchInfo li;
  int st = launch_info(kernel, NT, smem, li);
  if (st) return st;
  umma_residency<P, T, MODE>(li);
  const int64_t groups = (a.count + S::EPG - 1) / S::EPG;
  const int64_t need = (groups + S::GPC - 1) / S::GPC;
  const int64_t cap = (int64_t)li.grid_per_sm * li.num_sms;
  const int grid = (int)(need < cap ? need : cap);
  if (grid <= 0) return FEM_SUCCESS;
  kernel<<<grid, NT, smem, s>>>(a);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "assemble_kernel launch");
  return FEM_SUCCESS;
}

template <typename T, int MODE>
int launch_mode(int order, const dev::AsmArgs &a, cudaStream_t s) {
  switch (order) {
    case 1: return launch_p<1, T, MODE>(a, s);
    case 2: return launch_p<2, T, MODE>(a, s);
    case 3: return launch_p<3, T, MODE>(a, s);
    case 4: return launch_p<4, T, MODE>(a, s);
    default: return fail(FEM_ERR_INVALID_ORDER, "element order %d (supported: 1..4)", order);
  }
}

// The dispatchers below are defined out of line, each in the one translation unit
// that instantiates its kernels (every kernel is compiled once):
//   launch          single-mesh kernels, LINEAR (fem_kernels.cu), NONLINEAR via launch_nl
//   launch_nl       NONLINEAR kernels, FP64 (fem_nonlinear.cu)
//   launch_batched  tile-queue kernels of batches and the server (fem_batch.cu)
int launch(int order, int precision, int mode, const dev::AsmArgs &a, cudaStream_t s, int strain = FEM_STRAIN_LINEAR);
// Whether the order-4 MIXED element stiffness runs on the tcgen05 tensor cores (kU).
bool umma_order4();
int launch_nl(int order, int mode, const dev::AsmArgs &a, cudaStream_t s);
int launch_batched(int p, int precision, const dev::AsmArgs *meshes, const dev::Tile *tiles, int ntiles, int *counter,
                   cudaStream_t s);
// Order-1 row assembly (fem_rows.cu): chunks [a.begin, a.begin + a.count) of one
// mesh; or tiles of chunks of many meshes (residual and Jacobian).
int launch_rows(int mode, const dev::AsmArgs &a, cudaStream_t s);
int launch_rows_batched(const dev::AsmArgs *meshes, const dev::Tile *tiles, int ntiles, int *counter,
                        cudaStream_t s);
// Chunks per row tile of the batched row kernel.
constexpr int kRowTileChunks = 16;
// Warp-fragment kernel (fem_frag.cu): LINEAR assembly at orders 2 to 4 and NONLINEAR
// at orders 2 and 3 (frag_supported), plan mode (one colour, list positions
// [a.begin, a.begin + a.count)) or drop-in mode (elements through the reference map,
// accumulate-into).
// FEM_PRECISION_MIXED at order 3 runs its element stiffness as BF16x6 tensor-core
// products (b16_stiffness); the rest stays FP64.
bool frag_supported(int order, int precision, int strain, bool plan);
bool b16_stiffness(int order, int precision, int strain);
// chained: the launch directly follows this assembly's previous fragment-kernel
// launch on the stream and may overlap its tail (programmatic dependent launch).
int launch_frag(int order, int precision, int mode, const dev::AsmArgs &a, cudaStream_t s,
                int strain = FEM_STRAIN_LINEAR, bool chained = false);
// Its multi-range form (plan mode, residual always, Jacobian optional): up to
// kMaxRanges list-position ranges of one mesh in one launch.
int launch_frag_ranges(int order, int precision, int mode, const dev::AsmArgs &a, const dev::RangeList &r,
                       cudaStream_t s, int strain = FEM_STRAIN_LINEAR, bool chained = false);
// All colours of one plan in one dependency-ordered persistent launch (plan mode).
int launch_frag_sched(int order, int precision, int mode, const dev::AsmArgs &a, const dev::SchedArgs &sa,
                      cudaStream_t s, int strain = FEM_STRAIN_LINEAR);
// The batched colour launches of order p with an explicit kernel variant
// (FEM_KERNEL_FRAGMENT_* / FEM_KERNEL_ELEMENT_*).
int launch_batched_variant(int p, int variant, const dev::AsmArgs *meshes, const dev::Tile *tiles, int ntiles,
                           int *counter, cudaStream_t s);
// Its tile-queue form for batches and the server (residual and Jacobian).
int launch_frag_batched(int order, int precision, const dev::AsmArgs *meshes, const dev::Tile *tiles, int ntiles,
                        int *counter, cudaStream_t s);
// All colours of a batch's order-p meshes in one dependency-ordered persistent
// launch (sa.tiles name their meshes; residual and Jacobian).
int launch_frag_batched_sched(int order, int precision, const dev::AsmArgs *meshes, const dev::SchedArgs &sa,
                              cudaStream_t s);

// A synchronous cudaMemcpy from pageable host memory returns once the data is staged,
// before the DMA has landed, and a synchronous cudaMemset only enqueues; both run on
// the legacy default stream, which work on non-blocking streams (a caller's, the
// batch's, the server's) does not wait for.  Tables written that way are fenced with
// this before any kernel may read them.
inline int uploads_visible(const char *what) {
  const cudaError_t err = cudaStreamSynchronize(cudaStreamLegacy);
  return err == cudaSuccess ? (int)FEM_SUCCESS : cuda_fail(err, what);
}

inline void set_material(dev::AsmArgs &a, double E, double nu, double t) {
  // element/FEKernels.h:300-301
  a.mu = 0.5 * E / (1.0 + nu);
  a.lam = 2 * a.mu * nu / (1.0 - nu);
  a.t = t;
}

// Runs `body` on `stream`; with elapsed != NULL brackets it with events and synchronises.
template <typename F>
int timed(cudaStream_t s, double *elapsed, F body) {
  if (!elapsed) return body();
  cudaEvent_t e0, e1;
  cudaError_t err = cudaEventCreate(&e0);
  if (err != cudaSuccess) return cuda_fail(err, "cudaEventCreate");
  err = cudaEventCreate(&e1);
  if (err != cudaSuccess) {
    cudaEventDestroy(e0);
    return cuda_fail(err, "cudaEventCreate");
  }
  int st = FEM_SUCCESS;
  err = cudaEventRecord(e0, s);
  if (err != cudaSuccess) st = cuda_fail(err, "cudaEventRecord");
  if (!st) st = body();
  if (!st && (err = cudaEventRecord(e1, s)) != cudaSuccess) st = cuda_fail(err, "cudaEventRecord");
  if (!st && (err = cudaEventSynchronize(e1)) != cudaSuccess) st = cuda_fail(err, "kernel execution");
  float ms = 0.f;
  if (!st && (err = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) st = cuda_fail(err, "cudaEventElapsedTime");
  *elapsed = st ? 0.0 : ms * 1e-3;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

inline int epg_of(int p) {
  switch (p) {
    case 1: return dev::Shape<1>::EPG;
    case 2: return dev::Shape<2>::EPG;
    case 3: return dev::Shape<3>::EPG;
    default: return dev::Shape<4>::EPG;
  }
}

}  // namespace fem

// Device-resident topology of one mesh (see fem_plan_create).
struct fem_plan {
  int device = 0;
  int order = 0, nn = 0, numNodes = 0, numElements = 0, numColours = 0;
  int64_t nnzb = 0;
  std::vector<int> colourPtr;
  int *d_rowp = nullptr, *d_cols = nullptr, *d_connList = nullptr;
  uint8_t *d_blockCode = nullptr;  // per-element code records (Dims<P>::CS bytes each)
  // orders 2-4: pair layout of the fragment kernel's single-mesh colour launches
  // (HostPlan::pairColourPtr ...); usePairs selects it (fem_plan_set_layout)
  int *d_pairConnList = nullptr;
  uint8_t *d_pairCode = nullptr;
  std::vector<int> pairColourPtr, pairRegionEnd;
  std::vector<int> pairList, pairNodeLo, pairNodeHi;  // host copies for the band split of fem_plan_assemble_host
  int numPairColours = 0;
  int64_t numPairs = 0;
  bool usePairs = false;
  // order 1: row assembly tables (HostPlan::rowElemPtr/rowElem/rowChunk); numChunks == 0: none
  int *d_rowElemPtr = nullptr, *d_rowElem = nullptr, *d_rowChunk = nullptr;
  int numChunks = 0;
  // host side of the overlapped host-buffer assembly (fem_plan_assemble_host): the
  // colour-ordered element ids and each listed element's smallest and largest node
  std::vector<int> elemList, nodeLo, nodeHi;
  cudaStream_t copyIn = nullptr, copyOut = nullptr;  // created on first use
  int64_t deviceBytes = 0;
  int *d_waits = nullptr;  // bounded in-kernel waits of this plan's launches that ran out
  // dependency-ordered assembly (fem_plan_set_schedule): schedBand == 0 runs colour launches
  int schedBand = 0, schedTile = 0, schedGroups = 0, schedTiles = 0;
  void *d_sched = nullptr;  // one allocation: tiles, tiles per group, dependency CSR, status words
  fem::dev::SchedArgs sched{};
  int64_t schedBytes = 0;
};

namespace fem {
// The plan's device tables in an argument block (inputs/outputs/material are the caller's).
inline void plan_args(dev::AsmArgs &a, const fem_plan *p) {
  a.waits = p->d_waits;
  a.connList = p->d_connList;
  a.blockCode = p->d_blockCode;
  a.rowp = p->d_rowp;
  a.rowElemPtr = p->d_rowElemPtr;
  a.rowElem = p->d_rowElem;
  a.rowChunk = p->d_rowChunk;
}
// Whether the LINEAR assembly of this plan runs as row assembly.
inline bool plan_rows(const fem_plan *p) { return p->numChunks > 0; }
}  // namespace fem
