// fem_run_jacobian_batched_static: the batched drop-in Jacobian assembly for
// callers that cannot allocate device memory.
//
// Who cannot allocate: code that runs where cudaMalloc/cudaFree are off limits --
// inside a host callback or a real-time Newton loop that must not synchronise the
// device (cudaFree does), under a framework whose memory pool owns all device
// memory, or in a process whose device memory is already fully committed to
// resident meshes.  Such callers still own their inputs and outputs; what the
// batched kernel needs beyond them (the per-mesh argument table, the work-queue
// tiles and the queue counter) lives here, in one file-scope __device__ array.
//
// The array is loaded with the library and every GPU that loads it holds it until
// the process exits.  Host code cannot use the array's name as a device address
// (in host code it is a stand-in), so the first call on each device looks up the
// real address with cudaGetSymbolAddress while that device is current and caches
// it; that first call should be made before any stream capture.  The cached
// address belongs to the device's current context: after cudaDeviceReset the
// library must be reloaded.  All calls share the array and it keeps the last
// call's contents: the queue counter is cleared at the start of every call, and
// calls that overlap on the GPU race on it.
//
// The mesh table and tiles are staged in host arrays and copied with
// cudaMemcpyAsync from pageable memory, which CUDA may complete only after the
// work already queued on `stream` (the call can block the host until then).  A
// captured copy would read those host arrays again at every replay, after later
// calls had overwritten them, so calls on a stream that is being captured are
// refused with FEM_ERR_UNSUPPORTED.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "fem_common.h"
#include "fem_device.cuh"
#include "fem_launch.h"

namespace {

constexpr int kStaticMaxMeshes = 256;
constexpr int kStaticMaxTiles = 16384;
constexpr int kStaticTilesPerOrder = 3800;  // target; plus at most one short tile per mesh
constexpr int kMaxDevices = 64;

struct StaticLayout {
  static constexpr size_t args = 0;
  static constexpr size_t tiles = fem::dev::align16(args + sizeof(fem::dev::AsmArgs) * kStaticMaxMeshes);
  static constexpr size_t counters = fem::dev::align16(tiles + sizeof(fem::dev::Tile) * kStaticMaxTiles);
  static constexpr size_t total = fem::dev::align16(counters + sizeof(int) * 8);
};
static_assert(StaticLayout::total <= FEM_STATIC_SCRATCH_BYTES, "static scratch layout exceeds FEM_STATIC_SCRATCH_BYTES");

__device__ __align__(256) unsigned char g_static_scratch[FEM_STATIC_SCRATCH_BYTES];

std::mutex g_static_mu;
unsigned char *g_static_ptr[kMaxDevices] = {};

// Host staging of the table and tiles (pageable: cudaMemcpyAsync has copied it
// out before returning, so it is free again when the call returns).
fem::dev::AsmArgs g_host_args[kStaticMaxMeshes];
fem::dev::Tile g_host_tiles[kStaticMaxTiles];

int static_scratch(unsigned char **out) {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return fem::cuda_fail(err, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fem::fail(FEM_ERR_UNSUPPORTED, "device %d", dev);
  if (!g_static_ptr[dev]) {
    void *p = nullptr;
    err = cudaGetSymbolAddress(&p, g_static_scratch);
    if (err != cudaSuccess) return fem::cuda_fail(err, "cudaGetSymbolAddress(static scratch)");
    g_static_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_static_ptr[dev];
  return FEM_SUCCESS;
}

template <int P>
int launch_static_p(const fem::dev::AsmArgs *meshes, const fem::dev::Tile *tiles, int ntiles, int *counter,
                    cudaStream_t s) {
  using S = fem::dev::Shape<P>;
  constexpr int NT = S::GT * S::GPC;
  constexpr int MODE = fem::dev::kRes | fem::dev::kJac;
  auto kernel = fem::dev::assemble_batched_kernel<P, double, MODE>;
  const size_t smem = fem::dev::Layout<P, double, MODE>::total;
  fem::LaunchInfo li;
  int st = fem::launch_info(kernel, NT, smem, li);
  if (st) return st;
  const int64_t need = (ntiles + S::GPC - 1) / S::GPC;
  const int grid = (int)std::min<int64_t>(need, (int64_t)li.grid_per_sm * li.num_sms);
  if (grid <= 0) return FEM_SUCCESS;
  kernel<<<grid, NT, smem, s>>>(meshes, tiles, ntiles, counter);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return fem::cuda_fail(err, "static batched launch");
  return FEM_SUCCESS;
}

int launch_static(int p, const fem::dev::AsmArgs *meshes, const fem::dev::Tile *tiles, int ntiles, int *counter,
                  cudaStream_t s) {
  switch (p) {
    case 1: return launch_static_p<1>(meshes, tiles, ntiles, counter, s);
    case 2: return launch_static_p<2>(meshes, tiles, ntiles, counter, s);
    case 3: return launch_static_p<3>(meshes, tiles, ntiles, counter, s);
    default: return launch_static_p<4>(meshes, tiles, ntiles, counter, s);
  }
}

int epg_static(int p) {
  switch (p) {
    case 1: return fem::dev::Shape<1>::EPG;
    case 2: return fem::dev::Shape<2>::EPG;
    case 3: return fem::dev::Shape<3>::EPG;
    default: return fem::dev::Shape<4>::EPG;
  }
}

}  // namespace

extern "C" {

int fem_run_jacobian_batched_static(int numMeshes, const fem_dropin_mesh *meshes, void *stream) {
  fem::clear_error();
  if (numMeshes < 0 || (numMeshes > 0 && !meshes)) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "no mesh table");
  if (numMeshes > kStaticMaxMeshes)
    return fem::fail(FEM_ERR_UNSUPPORTED, "%d meshes exceed the static scratch limit of %d", numMeshes,
                     kStaticMaxMeshes);
  int64_t perOrder[5] = {0, 0, 0, 0, 0};
  for (int m = 0; m < numMeshes; m++) {
    const fem_dropin_mesh &d = meshes[m];
    if (d.elementOrder < 1 || d.elementOrder > 4)
      return fem::fail(FEM_ERR_INVALID_ORDER, "mesh %d: element order %d", m, d.elementOrder);
    if (d.numElements < 0) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "mesh %d: numElements < 0", m);
    if (d.numElements == 0) continue;
    if (!d.connPtr || !d.conn || !d.states || !d.nodeCoords || !d.elementBCSRMap || !d.residual || !d.matEntries)
      return fem::fail(FEM_ERR_INVALID_ARGUMENT, "mesh %d: NULL array", m);
    if (!fem::aligned16(d.states) || !fem::aligned16(d.nodeCoords) || !fem::aligned16(d.residual) ||
        (reinterpret_cast<uintptr_t>(d.matEntries) & 7u))
      return fem::fail(FEM_ERR_MISALIGNED, "mesh %d: vectors must be 16-byte aligned", m);
    perOrder[d.elementOrder] += d.numElements;
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t cerr = cudaStreamIsCapturing(s, &cap);
  if (cerr != cudaSuccess) return fem::cuda_fail(cerr, "cudaStreamIsCapturing");
  if (cap != cudaStreamCaptureStatusNone)
    return fem::fail(FEM_ERR_UNSUPPORTED, "the mesh table is staged from host memory at call time: "
                                          "calls on a capturing stream are refused");
  std::lock_guard<std::mutex> lk(g_static_mu);
  unsigned char *base = nullptr;
  int st = static_scratch(&base);
  if (st) return st;
  // Tile length per order: at least 16 element batches, long enough that the
  // order's tiles stay near kStaticTilesPerOrder.
  int64_t len[5] = {0, 0, 0, 0, 0};
  for (int p = 1; p <= 4; p++) {
    const int64_t minLen = 16 * (int64_t)epg_static(p);
    len[p] = std::max<int64_t>(minLen, (perOrder[p] + kStaticTilesPerOrder - 1) / kStaticTilesPerOrder);
    len[p] = (len[p] + epg_static(p) - 1) / epg_static(p) * epg_static(p);
  }
  int off[6] = {0, 0, 0, 0, 0, 0};
  int nt = 0;
  for (int p = 1; p <= 4; p++) {
    off[p] = nt;
    for (int m = 0; m < numMeshes; m++) {
      const fem_dropin_mesh &d = meshes[m];
      if (d.elementOrder != p) continue;
      for (int64_t k = 0; k < d.numElements; k += len[p]) {
        if (nt >= kStaticMaxTiles) return fem::fail(FEM_ERR_UNSUPPORTED, "work exceeds the static tile capacity");
        g_host_tiles[nt].mesh = m;
        g_host_tiles[nt].begin = k;
        g_host_tiles[nt].count = (int)std::min<int64_t>(len[p], d.numElements - k);
        nt++;
      }
    }
  }
  off[5] = nt;
  for (int m = 0; m < numMeshes; m++) {
    const fem_dropin_mesh &d = meshes[m];
    fem::dev::AsmArgs a{};
    a.connPtr = d.connPtr;
    a.conn = d.conn;
    a.map = d.elementBCSRMap;
    a.states = d.states;
    a.coords = d.nodeCoords;
    a.residual = d.residual;
    a.mat = d.matEntries;
    fem::set_material(a, d.E, d.nu, d.t);
    a.begin = 0;
    a.count = d.numElements;
    g_host_args[m] = a;
  }
  if (nt == 0) return FEM_SUCCESS;
  auto *d_args = reinterpret_cast<fem::dev::AsmArgs *>(base + StaticLayout::args);
  auto *d_tiles = reinterpret_cast<fem::dev::Tile *>(base + StaticLayout::tiles);
  int *d_counters = reinterpret_cast<int *>(base + StaticLayout::counters);
  cudaError_t err = cudaMemcpyAsync(d_args, g_host_args, sizeof(fem::dev::AsmArgs) * numMeshes,
                                    cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(d_tiles, g_host_tiles, sizeof(fem::dev::Tile) * nt, cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(d_counters, 0, sizeof(int) * 8, s);
  if (err != cudaSuccess) return fem::cuda_fail(err, "staging the static scratch");
  for (int p = 1; p <= 4; p++) {
    if (off[p + 1] <= off[p]) continue;
    st = launch_static(p, d_args, d_tiles + off[p], off[p + 1] - off[p], d_counters + p, s);
    if (st) return st;
  }
  return FEM_SUCCESS;
}

}  // extern "C"
