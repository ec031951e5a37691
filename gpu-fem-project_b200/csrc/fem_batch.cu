// Batched assembly of many meshes of mixed orders (fem_batch_*).
//
// Every mesh brings an assembly plan (colour-ordered elements, block codes).  The
// batch cuts each mesh's colour ranges into tiles and keeps one work queue per
// (order, colour): a tile list plus an atomic counter.  One persistent kernel per
// (order, colour) lets its groups pull tiles until the queue is empty, so meshes
// of very different sizes share the GPU without per-mesh launches.  Orders are
// independent chains on their own streams (colours of one order run in sequence:
// a later colour adds to blocks an earlier one stored); the whole fork/join
// pattern is captured once into a CUDA graph and replayed with one launch.
//
// Per order and precision the batch runs one kernel variant (FEM_KERNEL_*): the
// single-mesh plan path's kernel by default (batched results then equal the lone
// ones bit for bit), or one the autotuner picks by timing: the warp-fragment
// kernel (two elements per warp: 16 threads per element, 8 elements per 4-warp
// CTA step, FP64 MMA or, at order 3 MIXED, BF16x6 stiffness), the element kernel
// (one thread group per EPG elements: Shape<P> threads per group, groups per CTA;
// FP64 or, MIXED, FP32 element products, at order 4 MIXED also with its stiffness
// as BF16x6 tcgen05 MMAs), or order-1 row assembly.  MIXED may run
// any FP64 variant (FP64 is within its error bound); FP64 runs FP64 variants only.
// The tuner also picks the tile length of the order's work queues and, for the
// fragment kernels, whether an order's colours run as one launch each or all in
// one dependency-ordered persistent launch (fem_batch_set_ordered).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "fem_common.h"
#include "fem_device.cuh"
#include "fem_launch.h"

namespace fem {
namespace {

// One persistent batched launch of order P over the tile queue `tiles` (plan mode,
// residual and Jacobian).
template <int P, typename T>
int launch_batched_p(const dev::AsmArgs *meshes, const dev::Tile *tiles, int ntiles, int *counter, cudaStream_t s) {
  using S = dev::Shape<P>;
  constexpr int NT = S::GT * S::GPC;
  constexpr int MODE = dev::kPlan | dev::kRes | dev::kJac;
  auto kernel = dev::assemble_batched_kernel<P, T, MODE>;
  const size_t smem = dev::Layout<P, T, MODE>::total;
  LaunchInfo li;
  int st = launch_info(kernel, NT, smem, li);
  if (st) return st;
  const int64_t need = (ntiles + S::GPC - 1) / S::GPC;
  const int64_t cap = (int64_t)li.grid_per_sm * li.num_sms;
  const int grid = (int)(need < cap ? need : cap);
  if (grid <= 0) return FEM_SUCCESS;
  kernel<<<grid, NT, smem, s>>>(meshes, tiles, ntiles, counter);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "assemble_batched_kernel launch");
  return FEM_SUCCESS;
}

// The batched element kernel, every order, FP64 or FP32 element products.
template <typename T>
int launch_batched_t(int p, const dev::AsmArgs *meshes, const dev::Tile *tiles, int ntiles, int *counter,
                     cudaStream_t s) {
  switch (p) {
    case 1: return launch_batched_p<1, T>(meshes, tiles, ntiles, counter, s);
    case 2: return launch_batched_p<2, T>(meshes, tiles, ntiles, counter, s);
    case 3: return launch_batched_p<3, T>(meshes, tiles, ntiles, counter, s);
    case 4: return launch_batched_p<4, T>(meshes, tiles, ntiles, counter, s);
    default: return fail(FEM_ERR_INVALID_ORDER, "batched element kernel: order %d", p);
  }
}

// The batched order-4 element kernel with its stiffness on the tcgen05 tensor cores.
int launch_batched_umma(const dev::AsmArgs *meshes, const dev::Tile *tiles, int ntiles, int *counter,
                        cudaStream_t s) {
  using S = dev::Shape<4>;
  constexpr int NT = S::GT * S::GPC;
  constexpr int MODE = dev::kPlan | dev::kRes | dev::kJac | dev::kU;
  auto kernel = dev::assemble_batched_kernel<4, float, MODE>;
  const size_t smem = dev::Layout<4, float, MODE>::total;
  LaunchInfo li;
  int st = launch_info(kernel, NT, smem, li);
  if (st) return st;
  umma_residency<4, float, MODE>(li);
  const int64_t need = (ntiles + S::GPC - 1) / S::GPC;
  const int64_t cap = (int64_t)li.grid_per_sm * li.num_sms;
  const int grid = (int)(need < cap ? need : cap);
  if (grid <= 0) return FEM_SUCCESS;
  kernel<<<grid, NT, smem, s>>>(meshes, tiles, ntiles, counter);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, "assemble_batched_kernel (tcgen05) launch");
  return FEM_SUCCESS;
}

}  // namespace

// The colour launches of order p with kernel variant v (never FEM_KERNEL_DEFAULT
// or FEM_KERNEL_ROWS here).
int launch_batched_variant(int p, int v, const dev::AsmArgs *meshes, const dev::Tile *tiles, int ntiles, int *counter,
                           cudaStream_t s) {
  switch (v) {
    case FEM_KERNEL_FRAGMENT_FP64:
      return launch_frag_batched(p, FEM_PRECISION_FP64, meshes, tiles, ntiles, counter, s);
    case FEM_KERNEL_FRAGMENT_BF16X6:
      return launch_frag_batched(p, FEM_PRECISION_MIXED, meshes, tiles, ntiles, counter, s);
    case FEM_KERNEL_ELEMENT_FP64: return launch_batched_t<double>(p, meshes, tiles, ntiles, counter, s);
    case FEM_KERNEL_ELEMENT_FP32: return launch_batched_t<float>(p, meshes, tiles, ntiles, counter, s);
    case FEM_KERNEL_ELEMENT_TCGEN05:
      if (p != 4) return fail(FEM_ERR_INVALID_ARGUMENT, "tcgen05 element kernel: order 4 only");
      return launch_batched_umma(meshes, tiles, ntiles, counter, s);
    default: return fail(FEM_ERR_INVALID_ARGUMENT, "kernel variant %d", v);
  }
}

int launch_batched(int p, int precision, const dev::AsmArgs *meshes, const dev::Tile *tiles, int ntiles, int *counter,
                   cudaStream_t s) {
  // the same kernel as the single-mesh plan path, so batched results equal lone ones bit for bit
  if (frag_supported(p, precision, FEM_STRAIN_LINEAR, true))
    return launch_frag_batched(p, precision, meshes, tiles, ntiles, counter, s);
  if (precision == FEM_PRECISION_FP64) return launch_batched_t<double>(p, meshes, tiles, ntiles, counter, s);
  if (precision == FEM_PRECISION_MIXED && p == 4 && umma_order4())
    return launch_batched_umma(meshes, tiles, ntiles, counter, s);
  if (precision == FEM_PRECISION_MIXED) return launch_batched_t<float>(p, meshes, tiles, ntiles, counter, s);
  return fail(FEM_ERR_INVALID_ARGUMENT, "precision %d", precision);
}

}  // namespace fem

namespace {

constexpr int kMaxColours = 64;
constexpr int kOrders = 5;  // index 1..4

// Whether variant v may serve order p at `precision` (FEM_KERNEL_DEFAULT always may).
bool variant_allowed(int p, int precision, int v) {
  switch (v) {
    case FEM_KERNEL_DEFAULT: return true;
    case FEM_KERNEL_ROWS: return p == 1;
    case FEM_KERNEL_FRAGMENT_FP64: return p >= 2;
    case FEM_KERNEL_FRAGMENT_BF16X6: return p == 3 && precision == FEM_PRECISION_MIXED;
    case FEM_KERNEL_ELEMENT_FP64: return true;
    case FEM_KERNEL_ELEMENT_FP32: return precision == FEM_PRECISION_MIXED;
    case FEM_KERNEL_ELEMENT_TCGEN05: return p == 4 && precision == FEM_PRECISION_MIXED;
    default: return false;
  }
}

// The variant the single-mesh plan path runs for order p (order 1: rows where a
// mesh has row tables, the element kernel otherwise -- reported as ROWS).
int default_variant(int p, int precision) {
  if (p == 1) return FEM_KERNEL_ROWS;
  if (fem::frag_supported(p, precision, FEM_STRAIN_LINEAR, true))
    return fem::b16_stiffness(p, precision, FEM_STRAIN_LINEAR) ? FEM_KERNEL_FRAGMENT_BF16X6 : FEM_KERNEL_FRAGMENT_FP64;
  if (precision == FEM_PRECISION_MIXED)
    return p == 4 && fem::umma_order4() ? FEM_KERNEL_ELEMENT_TCGEN05 : FEM_KERNEL_ELEMENT_FP32;
  return FEM_KERNEL_ELEMENT_FP64;
}

int prec_index(int precision) { return precision == FEM_PRECISION_MIXED ? 1 : 0; }

}  // namespace

struct fem_batch {
  int device = 0;
  std::vector<const fem_plan *> plans;
  std::vector<fem::dev::AsmArgs> args;
  std::vector<char> bound;
  fem::dev::AsmArgs *d_args = nullptr;
  bool args_dirty = true;
  int maxColours = 0;
  int tileBatches[kOrders] = {0, 16, 16, 16, 16};  // tile length in element batches, per order
  int kernel[2][kOrders] = {};                       // [FP64, MIXED][order]: FEM_KERNEL_*
  std::vector<fem::dev::Tile> tiles;
  std::vector<int> tileOff;  // [kOrders][maxColours + 1]
  std::vector<int> rowSplit;  // order 1, per colour: tiles of meshes with row tables start here
  int rowTile0 = 0, rowTile1 = 0;  // order-1 row-assembly tiles (chunks), after the colour tiles
  fem::dev::Tile *d_tiles = nullptr;
  size_t d_tiles_cap = 0;
  bool tiles_dirty = true;
  int *d_counters = nullptr;  // [kOrders][kMaxColours]
  // per order: 1 = its colours in one dependency-ordered launch (fragment variants)
  int ordered[kOrders] = {};
  unsigned char *d_sched[kOrders] = {};
  fem::dev::SchedArgs sched[kOrders] = {};
  int schedGroups[kOrders] = {};
  int64_t schedBytes[kOrders] = {};
  bool sched_dirty = true;
  cudaStream_t streams[kOrders] = {};  // [0]: capture stream, [1..4]: one per order
  cudaEvent_t fork = nullptr, join[kOrders] = {};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graphPrecision = -1;
  int64_t totalElements = 0;
  int64_t deviceBytes = 0;
};

namespace {

void drop_graph(fem_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->graphPrecision = -1;
}

void batch_free(fem_batch *b) {
  if (!b) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  drop_graph(b);
  cudaFree(b->d_args);
  cudaFree(b->d_tiles);
  cudaFree(b->d_counters);
  for (int p = 0; p < kOrders; p++) cudaFree(b->d_sched[p]);
  for (int p = 0; p < kOrders; p++) {
    if (b->streams[p]) cudaStreamDestroy(b->streams[p]);
    if (b->join[p]) cudaEventDestroy(b->join[p]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  cudaSetDevice(cur);
  delete b;
}

int order_of(const fem_batch *b, int m) { return b->plans[m]->order; }

// Colour tiles of every mesh (order-1 meshes with row tables last within each
// colour, after rowSplit[c], so that row assembly can skip them) and the row
// tiles of the order-1 meshes that have row tables.
void build_tiles(fem_batch *b) {
  const int C = b->maxColours;
  b->tiles.clear();
  b->tileOff.assign((size_t)kOrders * (C + 1), 0);
  b->rowSplit.assign((size_t)C + 1, 0);
  for (int p = 1; p < kOrders; p++) {
    const int64_t len = (int64_t)b->tileBatches[p] * fem::epg_of(p);
    for (int c = 0; c < C; c++) {
      b->tileOff[p * (C + 1) + c] = (int)b->tiles.size();
      for (int rows = 0; rows < 2; rows++) {
        if (p == 1 && rows == 1) b->rowSplit[c] = (int)b->tiles.size();
        for (size_t m = 0; m < b->plans.size(); m++) {
          const fem_plan *pl = b->plans[m];
          if (pl->order != p || c >= pl->numColours || (int)fem::plan_rows(pl) != rows) continue;
          for (int64_t k = pl->colourPtr[c]; k < pl->colourPtr[c + 1]; k += len) {
            fem::dev::Tile t;
            t.mesh = (int)m;
            t.begin = k;
            t.count = (int)std::min<int64_t>(len, pl->colourPtr[c + 1] - k);
            b->tiles.push_back(t);
          }
        }
      }
    }
    b->tileOff[p * (C + 1) + C] = (int)b->tiles.size();
  }
  b->rowTile0 = (int)b->tiles.size();
  for (size_t m = 0; m < b->plans.size(); m++) {
    const fem_plan *pl = b->plans[m];
    if (!fem::plan_rows(pl)) continue;
    for (int k = 0; k < pl->numChunks; k += fem::kRowTileChunks) {
      fem::dev::Tile t;
      t.mesh = (int)m;
      t.begin = k;
      t.count = std::min(fem::kRowTileChunks, pl->numChunks - k);
      b->tiles.push_back(t);
    }
  }
  b->rowTile1 = (int)b->tiles.size();
  b->tiles_dirty = true;
  b->sched_dirty = true;
}

// The dependency-ordered launch of order p: one group per (mesh, colour), listed
// colours outermost (every mesh's colour 0, then every mesh's colour 1, ...), each
// cut into tiles of the order's tile length; a group waits for its mesh's previous
// colour, so every block still receives its contributions in colour order (the
// result equals the colour launches' bit for bit).  A warp holds only tiles it has
// pulled, in dispatch order, and every dependency is an earlier group: the
// earliest unfinished tile can always proceed.
int build_sched(fem_batch *b, int p) {
  cudaFree(b->d_sched[p]);
  b->d_sched[p] = nullptr;
  b->sched[p] = fem::dev::SchedArgs{};
  b->schedGroups[p] = 0;
  b->schedBytes[p] = 0;
  const int C = b->maxColours;
  const int64_t len = (int64_t)b->tileBatches[p] * fem::epg_of(p);
  std::vector<fem::dev::SchedTile> tiles;
  std::vector<int> groupTiles, depPtr(1, 0), deps, last(b->plans.size(), -1);
  for (int c = 0; c < C; c++)
    for (size_t m = 0; m < b->plans.size(); m++) {
      const fem_plan *pl = b->plans[m];
      if (pl->order != p || c >= pl->numColours || fem::plan_rows(pl)) continue;
      const int g = (int)groupTiles.size();
      int n = 0;
      for (int64_t k = pl->colourPtr[c]; k < pl->colourPtr[c + 1]; k += len, n++) {
        fem::dev::SchedTile t;
        t.begin = k;
        t.count = (int)std::min<int64_t>(len, pl->colourPtr[c + 1] - k);
        t.group = g;
        t.mesh = (int)m;
        tiles.push_back(t);
      }
      groupTiles.push_back(n);
      if (last[m] >= 0) deps.push_back(last[m]);
      depPtr.push_back((int)deps.size());
      last[m] = g;
    }
  const int G = (int)groupTiles.size();
  if (tiles.empty()) return FEM_SUCCESS;
  // one allocation: tiles | groupTiles | depPtr | deps | status (2 + G words)
  auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
  const size_t oT = 0, oG = al(oT + tiles.size() * sizeof(fem::dev::SchedTile)), oP = al(oG + 4 * (size_t)G),
               oD = al(oP + 4 * ((size_t)G + 1)), oS = al(oD + 4 * std::max<size_t>(deps.size(), 1)),
               total = oS + 4 * ((size_t)G + 2);
  cudaError_t err = cudaMalloc(&b->d_sched[p], total);
  if (err != cudaSuccess) return fem::cuda_fail(err, "cudaMalloc(batch schedule)");
  unsigned char *d = b->d_sched[p];
  err = cudaMemcpy(d + oT, tiles.data(), tiles.size() * sizeof(fem::dev::SchedTile), cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemcpy(d + oG, groupTiles.data(), 4 * (size_t)G, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemcpy(d + oP, depPtr.data(), 4 * ((size_t)G + 1), cudaMemcpyHostToDevice);
  if (err == cudaSuccess && !deps.empty()) err = cudaMemcpy(d + oD, deps.data(), 4 * deps.size(), cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemset(d + oS, 0, 4 * ((size_t)G + 2));
  if (err != cudaSuccess) return fem::cuda_fail(err, "batch schedule upload");
  fem::dev::SchedArgs &a = b->sched[p];
  a.tiles = reinterpret_cast<const fem::dev::SchedTile *>(d + oT);
  a.groupTiles = reinterpret_cast<const int *>(d + oG);
  a.depPtr = reinterpret_cast<const int *>(d + oP);
  a.deps = reinterpret_cast<const int *>(d + oD);
  a.status = reinterpret_cast<int *>(d + oS);
  a.ntiles = (int)tiles.size();
  a.stallGroup = -1;
  a.waitLimitNs = 500000000LL;
  b->schedGroups[p] = G;
  b->schedBytes[p] = (int64_t)total;
  return FEM_SUCCESS;
}

int sync_device_state(fem_batch *b) {
  cudaError_t err;
  const bool any = b->args_dirty || b->tiles_dirty || b->sched_dirty;
  if (b->sched_dirty) {
    for (int p = 2; p < kOrders; p++) {
      int st = b->ordered[p] ? build_sched(b, p) : FEM_SUCCESS;
      if (!b->ordered[p] && b->d_sched[p]) {
        cudaFree(b->d_sched[p]);
        b->d_sched[p] = nullptr;
        b->sched[p] = fem::dev::SchedArgs{};
        b->schedGroups[p] = 0;
        b->schedBytes[p] = 0;
      }
      if (st) return st;
    }
    b->sched_dirty = false;
  }
  if (b->args_dirty) {
    err = cudaMemcpy(b->d_args, b->args.data(), sizeof(fem::dev::AsmArgs) * b->args.size(), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) return fem::cuda_fail(err, "cudaMemcpy(mesh table)");
    b->args_dirty = false;
  }
  if (b->tiles_dirty) {
    const size_t need = std::max<size_t>(b->tiles.size(), 1);
    if (need > b->d_tiles_cap) {
      cudaFree(b->d_tiles);
      b->d_tiles = nullptr;
      err = cudaMalloc(&b->d_tiles, sizeof(fem::dev::Tile) * need);
      if (err != cudaSuccess) return fem::cuda_fail(err, "cudaMalloc(tiles)");
      b->d_tiles_cap = need;
    }
    if (!b->tiles.empty()) {
      err = cudaMemcpy(b->d_tiles, b->tiles.data(), sizeof(fem::dev::Tile) * b->tiles.size(),
                       cudaMemcpyHostToDevice);
      if (err != cudaSuccess) return fem::cuda_fail(err, "cudaMemcpy(tiles)");
    }
    b->tiles_dirty = false;
  }
  // the batch's launches run on non-blocking streams: the tables must have landed
  return any ? fem::uploads_visible("batch table upload") : (int)FEM_SUCCESS;
}

// The variant order p runs at `precision`.
int variant_of(const fem_batch *b, int p, int precision) {
  const int v = b->kernel[prec_index(precision)][p];
  return v == FEM_KERNEL_DEFAULT ? default_variant(p, precision) : v;
}

// The colour chain of one order on stream s (counters reset by the caller).  Order
// 1 with FEM_KERNEL_ROWS: one row-assembly launch (queue counter [0][0]) for the
// meshes with row tables, colour launches of the element kernel for the others.
// Whether order p runs its colours as one dependency-ordered launch with variant v.
bool sched_launch(const fem_batch *b, int p, int v) {
  const int C = b->maxColours;
  return p >= 2 && b->ordered[p] && b->tileOff[p * (C + 1) + C] > b->tileOff[p * (C + 1)] &&
         (v == FEM_KERNEL_FRAGMENT_FP64 || v == FEM_KERNEL_FRAGMENT_BF16X6);
}

int enqueue_order(fem_batch *b, int p, int precision, cudaStream_t s) {
  const int C = b->maxColours;
  const int v = variant_of(b, p, precision);
  if (sched_launch(b, p, v)) {
    if (b->sched[p].ntiles == 0) return FEM_SUCCESS;
    // the tile dispenser and group counters start at zero; the sticky count of
    // waits that ran out (word 0) is kept for fem_batch_wait_status
    cudaError_t err = cudaMemsetAsync(b->sched[p].status + 1, 0, sizeof(int) * ((size_t)b->schedGroups[p] + 1), s);
    if (err != cudaSuccess) return fem::cuda_fail(err, "cudaMemsetAsync(schedule counters)");
    return fem::launch_frag_batched_sched(p, v == FEM_KERNEL_FRAGMENT_BF16X6 ? FEM_PRECISION_MIXED : FEM_PRECISION_FP64,
                                          b->d_args, b->sched[p], s);
  }
  const bool rows = p == 1 && v == FEM_KERNEL_ROWS;
  if (rows && b->rowTile1 > b->rowTile0) {
    int st = fem::launch_rows_batched(b->d_args, b->d_tiles + b->rowTile0, b->rowTile1 - b->rowTile0,
                                      b->d_counters, s);
    if (st) return st;
  }
  for (int c = 0; c < C; c++) {
    const int t0 = b->tileOff[p * (C + 1) + c];
    const int t1 = rows ? b->rowSplit[c] : b->tileOff[p * (C + 1) + c + 1];
    if (t1 <= t0) continue;
    int *counter = b->d_counters + p * kMaxColours + c;
    int st = v == FEM_KERNEL_ROWS ? fem::launch_batched(p, precision, b->d_args, b->d_tiles + t0, t1 - t0, counter, s)
                                  : fem::launch_batched_variant(p, v, b->d_args, b->d_tiles + t0, t1 - t0, counter, s);
    if (st) return st;
  }
  return FEM_SUCCESS;
}

bool order_has_work(const fem_batch *b, int p) {
  const int C = b->maxColours;
  return b->tileOff[p * (C + 1) + C] > b->tileOff[p * (C + 1)];
}

// Whole batch: reset queues, fork one stream per order, join back into s.
int enqueue(fem_batch *b, int precision, cudaStream_t s) {
  cudaError_t err = cudaMemsetAsync(b->d_counters, 0, sizeof(int) * kOrders * kMaxColours, s);
  if (err != cudaSuccess) return fem::cuda_fail(err, "cudaMemsetAsync(counters)");
  if ((err = cudaEventRecord(b->fork, s)) != cudaSuccess) return fem::cuda_fail(err, "cudaEventRecord");
  for (int p = 1; p < kOrders; p++) {
    if (!order_has_work(b, p)) continue;
    if ((err = cudaStreamWaitEvent(b->streams[p], b->fork, 0)) != cudaSuccess)
      return fem::cuda_fail(err, "cudaStreamWaitEvent");
    int st = enqueue_order(b, p, precision, b->streams[p]);
    if (st) return st;
    if ((err = cudaEventRecord(b->join[p], b->streams[p])) != cudaSuccess)
      return fem::cuda_fail(err, "cudaEventRecord");
    if ((err = cudaStreamWaitEvent(s, b->join[p], 0)) != cudaSuccess)
      return fem::cuda_fail(err, "cudaStreamWaitEvent");
  }
  return FEM_SUCCESS;
}

int check_ready(fem_batch *b, int precision) {
  if (precision != FEM_PRECISION_FP64 && precision != FEM_PRECISION_MIXED)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "precision %d", precision);
  for (size_t m = 0; m < b->bound.size(); m++)
    if (!b->bound[m]) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "mesh %zu has no bound arrays", m);
  return sync_device_state(b);
}

}  // namespace

extern "C" {

int fem_batch_create(int numMeshes, fem_plan *const *plans, fem_batch **batch) {
  fem::clear_error();
  if (!batch) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "batch is NULL");
  *batch = nullptr;
  if (numMeshes <= 0 || !plans) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "no meshes");
  fem_batch *b = new fem_batch();
  cudaGetDevice(&b->device);
  for (int m = 0; m < numMeshes; m++) {
    if (!plans[m]) {
      delete b;
      return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan %d is NULL", m);
    }
    if (plans[m]->numColours > kMaxColours) {
      delete b;
      return fem::fail(FEM_ERR_UNSUPPORTED, "plan %d has %d colours (max %d)", m, plans[m]->numColours, kMaxColours);
    }
    b->plans.push_back(plans[m]);
    b->maxColours = std::max(b->maxColours, plans[m]->numColours);
    b->totalElements += plans[m]->numElements;
    fem::dev::AsmArgs a{};
    fem::plan_args(a, plans[m]);
    b->args.push_back(a);
  }
  b->bound.assign(numMeshes, 0);
  cudaError_t err = cudaMalloc(&b->d_args, sizeof(fem::dev::AsmArgs) * numMeshes);
  if (err == cudaSuccess) err = cudaMalloc(&b->d_counters, sizeof(int) * kOrders * kMaxColours);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (int p = 0; p < kOrders && err == cudaSuccess; p++) {
    err = cudaStreamCreateWithFlags(&b->streams[p], cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&b->join[p], cudaEventDisableTiming);
  }
  if (err != cudaSuccess) {
    int st = fem::cuda_fail(err, "fem_batch_create");
    batch_free(b);
    return st;
  }
  b->deviceBytes = (int64_t)(sizeof(fem::dev::AsmArgs) * numMeshes + sizeof(int) * kOrders * kMaxColours);
  build_tiles(b);
  *batch = b;
  return FEM_SUCCESS;
}

int fem_batch_destroy(fem_batch *batch) {
  fem::clear_error();
  batch_free(batch);
  return FEM_SUCCESS;
}

int fem_batch_bind(fem_batch *b, int mesh, const double *states, const double *nodeCoords, double E, double nu,
                   double t, double *residual, double *matEntries) {
  fem::clear_error();
  if (!b || mesh < 0 || mesh >= (int)b->plans.size()) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "bad mesh index");
  if (!states || !nodeCoords || !residual || !matEntries)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "batched meshes need states, coordinates, residual and matrix");
  if (!fem::aligned16(states) || !fem::aligned16(nodeCoords) || !fem::aligned16(residual) ||
      (reinterpret_cast<uintptr_t>(matEntries) & 31u))
    return fem::fail(FEM_ERR_MISALIGNED, "16-byte aligned vectors and a 32-byte aligned matrix are required");
  fem::dev::AsmArgs &a = b->args[mesh];
  a.states = states;
  a.coords = nodeCoords;
  a.residual = residual;
  a.mat = matEntries;
  fem::set_material(a, E, nu, t);
  a.begin = 0;
  a.count = b->plans[mesh]->numElements;
  b->bound[mesh] = 1;
  b->args_dirty = true;
  return FEM_SUCCESS;
}

int fem_batch_info(const fem_batch *b, int64_t *totalElements, int64_t *numTiles, int *numLaunches,
                   int64_t *deviceBytes) {
  fem::clear_error();
  if (!b) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (totalElements) *totalElements = b->totalElements;
  if (numTiles) *numTiles = (int64_t)b->tiles.size();
  if (numLaunches) {  // of an FP64 assembly with the batch's FP64 kernel variants
    int n = 0;
    const int C = b->maxColours;
    for (int p = 1; p < kOrders; p++) {
      if (sched_launch(b, p, variant_of(b, p, FEM_PRECISION_FP64))) {
        n++;
        continue;
      }
      const bool rows = p == 1 && variant_of(b, p, FEM_PRECISION_FP64) == FEM_KERNEL_ROWS;
      if (rows) n += b->rowTile1 > b->rowTile0;
      for (int c = 0; c < C; c++)
        n += (rows ? b->rowSplit[c] : b->tileOff[p * (C + 1) + c + 1]) > b->tileOff[p * (C + 1) + c];
    }
    *numLaunches = n;
  }
  if (deviceBytes) {
    *deviceBytes = b->deviceBytes + (int64_t)(sizeof(fem::dev::Tile) * b->d_tiles_cap);
    for (int p = 0; p < kOrders; p++) *deviceBytes += b->schedBytes[p];
  }
  return FEM_SUCCESS;
}

int fem_batch_get_tiles(const fem_batch *b, int *tileBatches) {
  fem::clear_error();
  if (!b || !tileBatches) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  for (int p = 1; p < kOrders; p++) tileBatches[p - 1] = b->tileBatches[p];
  return FEM_SUCCESS;
}

int fem_batch_set_tiles(fem_batch *b, const int *tileBatches) {
  fem::clear_error();
  if (!b || !tileBatches) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  for (int p = 1; p < kOrders; p++)
    if (tileBatches[p - 1] < 1) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "tile length must be >= 1");
  for (int p = 1; p < kOrders; p++) b->tileBatches[p] = tileBatches[p - 1];
  build_tiles(b);
  drop_graph(b);
  return FEM_SUCCESS;
}

int fem_batch_assemble(fem_batch *b, int precision, void *stream, double *elapsedSeconds) {
  fem::clear_error();
  if (elapsedSeconds) *elapsedSeconds = 0;
  if (!b) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "batch is NULL");
  int st = check_ready(b, precision);
  if (st) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return fem::timed(s, elapsedSeconds, [&] { return enqueue(b, precision, s); });
}

int fem_batch_capture(fem_batch *b, int precision, void *stream) {
  fem::clear_error();
  if (!b) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "batch is NULL");
  int st = check_ready(b, precision);
  if (st) return st;
  // The warm-up run sets the kernels' shared-memory attributes (not capturable)
  // after the caller's pending work on `stream`; the capture itself runs on the
  // batch's own stream (the legacy default stream cannot be captured).
  cudaStream_t user = reinterpret_cast<cudaStream_t>(stream);
  cudaStream_t s = b->streams[0];
  cudaError_t err = cudaEventRecord(b->join[0], user);
  if (err == cudaSuccess) err = cudaStreamWaitEvent(s, b->join[0], 0);
  if (err != cudaSuccess) return fem::cuda_fail(err, "ordering after the caller's stream");
  st = enqueue(b, precision, s);
  if (st) return st;
  err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return fem::cuda_fail(err, "warm-up before capture");
  drop_graph(b);
  err = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (err != cudaSuccess) return fem::cuda_fail(err, "cudaStreamBeginCapture");
  st = enqueue(b, precision, s);
  cudaGraph_t g = nullptr;
  err = cudaStreamEndCapture(s, &g);
  if (st) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (err != cudaSuccess) return fem::cuda_fail(err, "cudaStreamEndCapture");
  b->graph = g;
  err = cudaGraphInstantiate(&b->exec, g, 0);
  if (err != cudaSuccess) {
    drop_graph(b);
    return fem::cuda_fail(err, "cudaGraphInstantiate");
  }
  b->graphPrecision = precision;
  return FEM_SUCCESS;
}

int fem_batch_replay(fem_batch *b, void *stream, double *elapsedSeconds) {
  fem::clear_error();
  if (elapsedSeconds) *elapsedSeconds = 0;
  if (!b || !b->exec) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "no captured graph (call fem_batch_capture)");
  int st = sync_device_state(b);
  if (st) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return fem::timed(s, elapsedSeconds, [&] {
    cudaError_t err = cudaGraphLaunch(b->exec, s);
    return err == cudaSuccess ? (int)FEM_SUCCESS : fem::cuda_fail(err, "cudaGraphLaunch");
  });
}

int fem_batch_get_kernels(const fem_batch *b, int precision, int *kernels) {
  fem::clear_error();
  if (!b || !kernels) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  if (precision != FEM_PRECISION_FP64 && precision != FEM_PRECISION_MIXED)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "precision %d", precision);
  for (int p = 1; p < kOrders; p++) kernels[p - 1] = variant_of(b, p, precision);
  return FEM_SUCCESS;
}

int fem_batch_set_kernels(fem_batch *b, int precision, const int *kernels) {
  fem::clear_error();
  if (!b || !kernels) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  if (precision != FEM_PRECISION_FP64 && precision != FEM_PRECISION_MIXED)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "precision %d", precision);
  for (int p = 1; p < kOrders; p++)
    if (!variant_allowed(p, precision, kernels[p - 1]))
      return fem::fail(FEM_ERR_INVALID_ARGUMENT, "kernel %d cannot serve order %d at precision %d", kernels[p - 1], p,
                       precision);
  for (int p = 1; p < kOrders; p++) b->kernel[prec_index(precision)][p] = kernels[p - 1];
  drop_graph(b);
  return FEM_SUCCESS;
}

int fem_batch_set_ordered(fem_batch *b, const int *ordered) {
  fem::clear_error();
  if (!b || !ordered) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  if (ordered[0] != 0) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "order 1 has no dependency-ordered launch");
  for (int p = 2; p < kOrders; p++) b->ordered[p] = ordered[p - 1] != 0;
  b->sched_dirty = true;
  drop_graph(b);
  return FEM_SUCCESS;
}

int fem_batch_get_ordered(const fem_batch *b, int *ordered) {
  fem::clear_error();
  if (!b || !ordered) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  for (int p = 1; p < kOrders; p++) ordered[p - 1] = b->ordered[p];
  return FEM_SUCCESS;
}

int fem_batch_wait_status(fem_batch *b, void *stream, int64_t *timedOutWaits) {
  fem::clear_error();
  if (!b || !timedOutWaits) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  *timedOutWaits = 0;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int v[kOrders] = {};
  cudaError_t err = cudaSuccess;
  for (int p = 2; p < kOrders && err == cudaSuccess; p++)
    if (b->d_sched[p]) err = cudaMemcpyAsync(&v[p], b->sched[p].status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  for (int p = 2; p < kOrders && err == cudaSuccess; p++)
    if (v[p]) err = cudaMemsetAsync(b->sched[p].status, 0, sizeof(int), s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return fem::cuda_fail(err, "reading the batch's wait status");
  for (int p = 2; p < kOrders; p++) *timedOutWaits += v[p];
  return FEM_SUCCESS;
}

int fem_batch_set_schedule_waits(fem_batch *b, int64_t waitLimitNs, int order, int stallGroup) {
  fem::clear_error();
  if (!b) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (order < 2 || order > 4) return fem::fail(FEM_ERR_INVALID_ORDER, "order %d", order);
  int st = sync_device_state(b);
  if (st) return st;
  if (stallGroup != -1 && (stallGroup < 0 || stallGroup >= b->schedGroups[order]))
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "stallGroup %d of %d groups", stallGroup, b->schedGroups[order]);
  if (waitLimitNs > 0) b->sched[order].waitLimitNs = waitLimitNs;
  b->sched[order].stallGroup = stallGroup;
  drop_graph(b);
  return FEM_SUCCESS;
}

int fem_batch_tune(fem_batch *b, int precision, void *stream, int reps, double *bestSeconds) {
  fem::clear_error();
  if (!b) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (reps < 1) reps = 1;
  int st = check_ready(b, precision);
  if (st) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  static const int lens[] = {1, 4, 16, 64, 256};
  static const int variants[] = {FEM_KERNEL_ROWS, FEM_KERNEL_FRAGMENT_FP64, FEM_KERNEL_FRAGMENT_BF16X6,
                                 FEM_KERNEL_ELEMENT_FP64, FEM_KERNEL_ELEMENT_FP32, FEM_KERNEL_ELEMENT_TCGEN05};
  int *kern = b->kernel[prec_index(precision)];
  double total = 0;
  for (int p = 1; p < kOrders; p++) {
    if (!order_has_work(b, p)) continue;
    double best = 1e30;
    int bestLen = b->tileBatches[p], bestVar = kern[p], bestOrd = b->ordered[p];
    for (int v : variants) {
      if (!variant_allowed(p, precision, v)) continue;
      kern[p] = v;
      const bool frag = v == FEM_KERNEL_FRAGMENT_FP64 || v == FEM_KERNEL_FRAGMENT_BF16X6;
      for (int ord = 0; ord <= (frag && p >= 2 ? 1 : 0); ord++)
      for (int len : lens) {
        b->ordered[p] = ord;
        b->tileBatches[p] = len;
        build_tiles(b);
        if ((st = sync_device_state(b))) return st;
        double secs = 0;
        for (int r = 0; r <= reps; r++) {  // first run warms up
          double one = 0;
          st = fem::timed(s, &one, [&] {
            cudaError_t err = cudaMemsetAsync(b->d_counters, 0, sizeof(int) * kOrders * kMaxColours, s);
            if (err != cudaSuccess) return fem::cuda_fail(err, "cudaMemsetAsync");
            return enqueue_order(b, p, precision, s);
          });
          if (st) return st;
          if (r > 0) secs += one;
        }
        secs /= reps;
        if (secs < best) {
          best = secs;
          bestLen = len;
          bestVar = v;
          bestOrd = ord;
        }
      }
    }
    b->tileBatches[p] = bestLen;
    kern[p] = bestVar;
    b->ordered[p] = bestOrd;
    total += best;
  }
  build_tiles(b);
  drop_graph(b);
  if (bestSeconds) *bestSeconds = total;
  return sync_device_state(b);
}

}  // extern "C"
