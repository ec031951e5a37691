// Assembly server: continuous batching of residual + Jacobian requests from many
// independent Newton solves over device-resident meshes (fem_server_*).
//
// Clients register a mesh once (plan, coordinates, state, residual and matrix
// stay on the device; admission is refused with FEM_ERR_BUDGET when the device
// bytes would exceed the server's budget) and then submit requests, each with a
// new host state and a host buffer for the residual.  A dispatcher thread takes
// pending requests whenever one of the server's kLanes lanes is free: the small
// ones (meshes of at most kSmallRequest elements) first, in arrival order, up to
// kSmallWave elements, so that a small request never waits inside a large wave;
// else all of them in arrival order (also once the oldest has waited kMaxWait),
// up to maxBatch requests and, past the first one, kWaveElements elements.  It
// issues on that lane's stream: the wave's mesh table and tile list, the state
// copies, one batched persistent launch per (order, colour) over the requested
// meshes' tiles, and the residual copies, smallest first, each followed by an
// event of its request.  Each lane has a high- and a low-priority stream: waves
// of at most kSmallWave elements run on the high-priority one, so that the block
// scheduler starts their kernels ahead of the queued launches of larger waves.  Requests that arrive while
// lanes are busy go to the next free lane, so waves overlap on the device; a
// waiter thread per lane completes each request as soon as its own residual has
// arrived.  Results do not depend on which requests share a wave (see the batched
// kernel: every block receives exactly one contribution per colour).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "fem_common.h"
#include "fem_device.cuh"
#include "fem_launch.h"

namespace {

// Lanes (concurrent waves): 8 measured best for 64 clients (4: lower saturated
// throughput and a longer tail; 12 and 16: no better)
constexpr int kLanes = 8;
constexpr int kMaxColoursS = 64;
constexpr int64_t kWaveElements = 1 << 21;  // element cap of a wave past its first request
constexpr int64_t kSmallRequest = 1 << 15;  // requests taken first
constexpr int64_t kSmallWave = 1 << 17;     // waves up to this many elements run at high priority
constexpr double kMaxWait = 0.01;           // seconds: past this the oldest request goes first

double now_seconds() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct ServerMesh {
  fem_plan *plan = nullptr;
  double *coords = nullptr, *states = nullptr, *residual = nullptr, *mat = nullptr;
  int64_t bytes = 0;
  double E = 0, nu = 0, t = 0;
  bool busy = false;  // a request of this mesh is queued or running
};

struct Request {
  int mesh = -1;
  const double *hostStates = nullptr;
  double *hostResidual = nullptr;
  double tSubmit = 0, tDone = 0;
  int status = FEM_SUCCESS;
  bool done = false;
};

struct Lane {
  cudaStream_t stream = nullptr;  // the current wave's stream: hi or lo
  cudaStream_t hi = nullptr, lo = nullptr;
  cudaEvent_t done = nullptr;
  std::vector<cudaEvent_t> reqDone;  // per request of the wave, after its residual copy (maxBatch events)
  std::vector<int> doneOrder;        // wave positions in the order their events were recorded
  fem::dev::AsmArgs *d_args = nullptr;
  fem::dev::Tile *d_tiles = nullptr;
  int *d_counters = nullptr;
  size_t argsCap = 0, tilesCap = 0;
  std::vector<fem::dev::AsmArgs> args;
  std::vector<fem::dev::Tile> tiles;
  std::vector<int64_t> reqs;
  bool busy = false;    // reserved by the dispatcher for a wave
  bool issued = false;  // the wave's work is on the stream and L.done recorded after it
  std::thread waiter;
  std::condition_variable cv;
};

}  // namespace

struct fem_server {
  int device = 0;
  int precision = FEM_PRECISION_FP64;
  int maxBatch = 64;
  int64_t budget = 0, used = 0;
  int tileBatches = 16;
  std::mutex mu;
  std::condition_variable cvDispatch, cvDone;
  std::vector<ServerMesh> meshes;
  std::unordered_map<int64_t, Request> reqs;
  std::deque<int64_t> pending;
  int64_t nextTicket = 1;
  int64_t maxMeshElements = 0;  // largest registered mesh
  int maxMeshColours = 0;
  Lane lanes[kLanes];
  std::thread dispatcher;
  bool stop = false;
  // statistics
  int64_t waves = 0, completed = 0, elementsDone = 0;
};

namespace {

int lane_reserve(Lane &L, size_t nargs, size_t ntiles) {
  cudaError_t err;
  if (nargs > L.argsCap) {
    cudaFree(L.d_args);
    L.d_args = nullptr;
    L.argsCap = std::max<size_t>(nargs, 2 * L.argsCap);
    if ((err = cudaMalloc(&L.d_args, sizeof(fem::dev::AsmArgs) * L.argsCap)) != cudaSuccess)
      return fem::cuda_fail(err, "cudaMalloc(lane args)");
  }
  if (ntiles > L.tilesCap) {
    cudaFree(L.d_tiles);
    L.d_tiles = nullptr;
    L.tilesCap = std::max<size_t>(ntiles, 2 * L.tilesCap);
    if ((err = cudaMalloc(&L.d_tiles, sizeof(fem::dev::Tile) * L.tilesCap)) != cudaSuccess)
      return fem::cuda_fail(err, "cudaMalloc(lane tiles)");
  }
  return FEM_SUCCESS;
}

// Upper bound of the tiles of one wave: at most maxBatch meshes and, past its first
// request, kWaveElements elements (a single request may exceed it); per mesh and
// colour one partial tile beyond elements / tile length; order-1 row tiles hold
// kRowTileChunks chunks of up to kRowChunkRows rows (at least one element per
// chunk row band), plus one partial tile per mesh.
size_t lane_tile_bound(const fem_server *S) {
  const int64_t ne = std::max<int64_t>(kWaveElements, S->maxMeshElements);
  const int64_t perTile = std::max<int64_t>(1, S->tileBatches);  // the smallest tile: EPG >= 1
  return (size_t)(ne / perTile + ne / fem::kRowTileChunks + (int64_t)S->maxBatch * (S->maxMeshColours + 2) + 1);
}

// Issues one wave on lane L (called by the dispatcher without the server lock;
// the wave's requests are owned by the lane until its waiter completes them).
int issue_wave(fem_server *S, Lane &L, const std::vector<ServerMesh> &wm, const std::vector<Request *> &rq) {
  cudaError_t err;
  const int n = (int)wm.size();
  L.args.resize(n);
  int maxC = 0;
  for (int i = 0; i < n; i++) {
    const ServerMesh &m = wm[i];
    fem::dev::AsmArgs a{};
    fem::plan_args(a, m.plan);
    a.states = m.states;
    a.coords = m.coords;
    a.residual = m.residual;
    a.mat = m.mat;
    fem::set_material(a, m.E, m.nu, m.t);
    a.begin = 0;
    a.count = m.plan->numElements;
    L.args[i] = a;
    maxC = std::max(maxC, m.plan->numColours);
  }
  // tiles grouped by (order, colour)
  L.tiles.clear();
  std::vector<int> off;
  std::vector<std::pair<int, int>> keys;
  for (int p = 1; p <= 4; p++) {
    const int64_t len = (int64_t)S->tileBatches * fem::epg_of(p);
    for (int c = 0; c < maxC; c++) {
      const int t0 = (int)L.tiles.size();
      for (int i = 0; i < n; i++) {
        const fem_plan *pl = wm[i].plan;
        if (pl->order != p || c >= pl->numColours || fem::plan_rows(pl)) continue;
        for (int64_t k = pl->colourPtr[c]; k < pl->colourPtr[c + 1]; k += len) {
          fem::dev::Tile t;
          t.mesh = i;
          t.begin = k;
          t.count = (int)std::min<int64_t>(len, pl->colourPtr[c + 1] - k);
          L.tiles.push_back(t);
        }
      }
      if ((int)L.tiles.size() > t0) {
        keys.push_back({p, c});
        off.push_back(t0);
      }
    }
  }
  // order-1 meshes with row tables: one row-assembly launch (key colour -1)
  {
    const int t0 = (int)L.tiles.size();
    for (int i = 0; i < n; i++) {
      const fem_plan *pl = wm[i].plan;
      if (!fem::plan_rows(pl)) continue;
      for (int k = 0; k < pl->numChunks; k += fem::kRowTileChunks) {
        fem::dev::Tile t;
        t.mesh = i;
        t.begin = k;
        t.count = std::min(fem::kRowTileChunks, pl->numChunks - k);
        L.tiles.push_back(t);
      }
    }
    if ((int)L.tiles.size() > t0) {
      keys.push_back({1, -1});
      off.push_back(t0);
    }
  }
  off.push_back((int)L.tiles.size());
  int st = lane_reserve(L, n, std::max<size_t>(L.tiles.size(), 1));
  if (st) return st;
  int64_t waveElements = 0;
  for (int i = 0; i < n; i++) waveElements += wm[i].plan->numElements;
  L.stream = waveElements <= kSmallWave ? L.hi : L.lo;
  // The mesh table and tile list come from pageable vectors: a pageable upload
  // first waits for the stream's earlier work, so it goes before the state
  // uploads, on the lane's idle stream (after them it would hold the dispatcher
  // until the states had crossed PCIe).
  err = cudaMemcpyAsync(L.d_args, L.args.data(), sizeof(fem::dev::AsmArgs) * n, cudaMemcpyHostToDevice, L.stream);
  if (err == cudaSuccess && !L.tiles.empty())
    err = cudaMemcpyAsync(L.d_tiles, L.tiles.data(), sizeof(fem::dev::Tile) * L.tiles.size(), cudaMemcpyHostToDevice,
                          L.stream);
  if (err == cudaSuccess)
    err = cudaMemsetAsync(L.d_counters, 0, sizeof(int) * 5 * kMaxColoursS, L.stream);
  if (err != cudaSuccess) return fem::cuda_fail(err, "wave staging");
  // inputs: new states
  for (int i = 0; i < n; i++) {
    const ServerMesh &m = wm[i];
    err = cudaMemcpyAsync(m.states, rq[i]->hostStates, sizeof(double) * 2 * m.plan->numNodes, cudaMemcpyHostToDevice,
                          L.stream);
    if (err != cudaSuccess) return fem::cuda_fail(err, "state upload");
  }
  for (size_t j = 0; j < keys.size(); j++) {
    const int p = keys[j].first, c = keys[j].second;
    if (c < 0) {  // row assembly, queue counter [0][0]
      st = fem::launch_rows_batched(L.d_args, L.d_tiles + off[j], off[j + 1] - off[j], L.d_counters, L.stream);
      if (st) return st;
      continue;
    }
    int *counter = L.d_counters + p * kMaxColoursS + c;
    st = fem::launch_batched(p, S->precision, L.d_args, L.d_tiles + off[j], off[j + 1] - off[j], counter, L.stream);
    if (st) return st;
  }
  // outputs: residuals back to the clients, smallest first, each request's event
  // after its own copy (the matrices stay resident)
  L.doneOrder.resize(n);
  for (int i = 0; i < n; i++) L.doneOrder[i] = i;
  auto bytes_of = [&](int i) { return rq[i]->hostResidual ? (int64_t)wm[i].plan->numNodes : (int64_t)-1; };
  std::stable_sort(L.doneOrder.begin(), L.doneOrder.end(), [&](int a, int b) { return bytes_of(a) < bytes_of(b); });
  for (int j = 0; j < n; j++) {
    const int i = L.doneOrder[j];
    const ServerMesh &m = wm[i];
    if (rq[i]->hostResidual) {
      err = cudaMemcpyAsync(rq[i]->hostResidual, m.residual, sizeof(double) * 2 * m.plan->numNodes,
                            cudaMemcpyDeviceToHost, L.stream);
      if (err != cudaSuccess) return fem::cuda_fail(err, "residual download");
    }
    if ((err = cudaEventRecord(L.reqDone[j], L.stream)) != cudaSuccess) return fem::cuda_fail(err, "cudaEventRecord");
  }
  err = cudaEventRecord(L.done, L.stream);
  if (err != cudaSuccess) return fem::cuda_fail(err, "cudaEventRecord");
  return FEM_SUCCESS;
}

void dispatcher_main(fem_server *S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  while (true) {
    int free_lane = -1;
    S->cvDispatch.wait(lk, [&] {
      if (S->stop) return true;
      if (S->pending.empty()) return false;
      for (int l = 0; l < kLanes; l++)
        if (!S->lanes[l].busy) {
          free_lane = l;
          return true;
        }
      return false;
    });
    if (S->stop) return;
    Lane &L = S->lanes[free_lane];
    // copies of the wave's mesh records: the mesh vector may grow while the
    // wave is issued without the lock (the meshes themselves stay put: a mesh
    // with a request in flight cannot be removed)
    std::vector<ServerMesh> wm;
    std::vector<Request *> rq;
    L.reqs.clear();
    auto elements_of = [&](int64_t tk) { return S->meshes[S->reqs[tk].mesh].plan->numElements; };
    bool smallFirst = false;
    if (now_seconds() - S->reqs[S->pending.front()].tSubmit < kMaxWait)
      for (int64_t tk : S->pending)
        if (elements_of(tk) <= kSmallRequest) {
          smallFirst = true;
          break;
        }
    int64_t waveElements = 0;
    for (auto it = S->pending.begin(); it != S->pending.end() && (int)L.reqs.size() < S->maxBatch;) {
      const int64_t tk = *it;
      const int64_t ne = elements_of(tk);
      if (smallFirst && ne > kSmallRequest) {
        ++it;
        continue;
      }
      if (!L.reqs.empty() && waveElements + ne > (smallFirst ? kSmallWave : kWaveElements)) break;
      waveElements += ne;
      it = S->pending.erase(it);
      Request &r = S->reqs[tk];
      L.reqs.push_back(tk);
      wm.push_back(S->meshes[r.mesh]);
      rq.push_back(&r);
    }
    L.busy = true;
    S->waves++;
    lk.unlock();
    int st = issue_wave(S, L, wm, rq);
    // a failed wave may have left work on its stream; the lane's next wave (on
    // either stream) reuses the mesh table and tile buffers
    if (st) cudaStreamSynchronize(L.stream);
    lk.lock();
    if (st) {
      for (int64_t tk : L.reqs) {
        Request &r = S->reqs[tk];
        r.status = st;
        r.done = true;
        r.tDone = now_seconds();
        S->meshes[r.mesh].busy = false;
      }
      L.reqs.clear();
      L.busy = false;
      S->cvDone.notify_all();
      continue;
    }
    L.issued = true;
    L.cv.notify_all();
  }
}

void waiter_main(fem_server *S, int l) {
  cudaSetDevice(S->device);
  Lane &L = S->lanes[l];
  std::unique_lock<std::mutex> lk(S->mu);
  while (true) {
    L.cv.wait(lk, [&] { return S->stop || L.issued; });
    if (S->stop) return;
    // each request completes as soon as its own residual has arrived
    for (size_t j = 0; j < L.reqs.size(); j++) {
      lk.unlock();
      const cudaError_t err = cudaEventSynchronize(L.reqDone[j]);
      const double t = now_seconds();
      lk.lock();
      Request &r = S->reqs[L.reqs[L.doneOrder[j]]];
      r.status = err == cudaSuccess ? FEM_SUCCESS : FEM_ERR_CUDA;
      r.done = true;
      r.tDone = t;
      S->meshes[r.mesh].busy = false;
      S->completed++;
      S->elementsDone += S->meshes[r.mesh].plan->numElements;
      S->cvDone.notify_all();
    }
    lk.unlock();
    const cudaError_t err = cudaEventSynchronize(L.done);
    lk.lock();
    (void)err;
    L.reqs.clear();
    L.issued = false;
    L.busy = false;
    S->cvDone.notify_all();
    S->cvDispatch.notify_all();
  }
}

void server_free(fem_server *S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cvDispatch.notify_all();
  for (auto &L : S->lanes) L.cv.notify_all();
  if (S->dispatcher.joinable()) S->dispatcher.join();
  for (auto &L : S->lanes)
    if (L.waiter.joinable()) L.waiter.join();
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(S->device);
  for (auto &L : S->lanes) {
    if (L.hi) cudaStreamSynchronize(L.hi);
    if (L.lo) cudaStreamSynchronize(L.lo);
    cudaFree(L.d_args);
    cudaFree(L.d_tiles);
    cudaFree(L.d_counters);
    if (L.done) cudaEventDestroy(L.done);
    for (cudaEvent_t e : L.reqDone) cudaEventDestroy(e);
    if (L.hi) cudaStreamDestroy(L.hi);
    if (L.lo) cudaStreamDestroy(L.lo);
  }
  for (auto &m : S->meshes) {
    if (!m.plan) continue;
    cudaFree(m.coords);
    cudaFree(m.states);
    cudaFree(m.residual);
    cudaFree(m.mat);
    fem_plan_destroy(m.plan);
  }
  cudaSetDevice(cur);
  delete S;
}

}  // namespace

extern "C" {

int fem_server_create(int64_t budgetBytes, int precision, int maxBatch, fem_server **server) {
  fem::clear_error();
  if (!server) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "server is NULL");
  *server = nullptr;
  if (budgetBytes <= 0 || maxBatch < 1) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "budget and maxBatch must be > 0");
  if (precision != FEM_PRECISION_FP64 && precision != FEM_PRECISION_MIXED)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "precision %d", precision);
  fem_server *S = new fem_server();
  cudaGetDevice(&S->device);
  S->budget = budgetBytes;
  S->precision = precision;
  S->maxBatch = maxBatch;
  int leastPri = 0, greatestPri = 0;
  cudaError_t err = cudaDeviceGetStreamPriorityRange(&leastPri, &greatestPri);
  for (auto &L : S->lanes) {
    if (err == cudaSuccess) err = cudaStreamCreateWithPriority(&L.hi, cudaStreamNonBlocking, greatestPri);
    if (err == cudaSuccess) err = cudaStreamCreateWithPriority(&L.lo, cudaStreamNonBlocking, leastPri);
    L.stream = L.lo;
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming);
    if (err == cudaSuccess) err = cudaMalloc(&L.d_counters, sizeof(int) * 5 * kMaxColoursS);
    L.reqDone.assign((size_t)maxBatch, nullptr);
    for (auto &e : L.reqDone)
      if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  }
  if (err != cudaSuccess) {
    int st = fem::cuda_fail(err, "fem_server_create");
    server_free(S);
    return st;
  }
  S->dispatcher = std::thread(dispatcher_main, S);
  for (int l = 0; l < kLanes; l++) S->lanes[l].waiter = std::thread(waiter_main, S, l);
  *server = S;
  return FEM_SUCCESS;
}

int fem_server_destroy(fem_server *server) {
  fem::clear_error();
  server_free(server);
  return FEM_SUCCESS;
}

int fem_server_add_mesh(fem_server *S, int elementOrder, int numNodes, const int *connPtr, const int *conn,
                        int numElements, const double *nodeCoords, double E, double nu, double t, int *meshId) {
  fem::clear_error();
  if (!S || !meshId || !nodeCoords) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  fem_plan *plan = nullptr;
  int st = fem_plan_create(elementOrder, numNodes, connPtr, conn, numElements, &plan);
  if (st) return st;
  const int64_t vec = (int64_t)sizeof(double) * 2 * numNodes;
  const int64_t bytes = plan->deviceBytes + 3 * vec + 32 * plan->nnzb;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->used + bytes > S->budget) {
      fem_plan_destroy(plan);
      return fem::fail(FEM_ERR_BUDGET, "mesh needs %lld bytes, %lld of %lld in use", (long long)bytes,
                       (long long)S->used, (long long)S->budget);
    }
    S->used += bytes;
  }
  ServerMesh m;
  m.plan = plan;
  m.bytes = bytes;
  m.E = E;
  m.nu = nu;
  m.t = t;
  cudaError_t err = cudaMalloc(&m.coords, vec);
  if (err == cudaSuccess) err = cudaMalloc(&m.states, vec);
  if (err == cudaSuccess) err = cudaMalloc(&m.residual, vec);
  if (err == cudaSuccess) err = cudaMalloc(&m.mat, 32 * plan->nnzb + 32);
  if (err == cudaSuccess) err = cudaMemcpy(m.coords, nodeCoords, vec, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemset(m.states, 0, vec);
  // the lanes' streams do not wait for the legacy stream's copy and clear
  if (err == cudaSuccess) err = cudaStreamSynchronize(cudaStreamLegacy);
  if (err != cudaSuccess) {
    cudaFree(m.coords);
    cudaFree(m.states);
    cudaFree(m.residual);
    cudaFree(m.mat);
    fem_plan_destroy(plan);
    std::lock_guard<std::mutex> lk(S->mu);
    S->used -= bytes;
    return fem::cuda_fail(err, "fem_server_add_mesh");
  }
  std::lock_guard<std::mutex> lk(S->mu);
  // Size the idle lanes' mesh tables and tile lists for any wave the meshes
  // registered so far can form, so that serving never allocates: a cudaFree in
  // the dispatcher would synchronise the device under every lane's running wave.
  S->maxMeshElements = std::max<int64_t>(S->maxMeshElements, numElements);
  S->maxMeshColours = std::max(S->maxMeshColours, plan->numColours);
  const size_t tiles = lane_tile_bound(S);
  for (auto &L : S->lanes)
    if (!L.busy && (st = lane_reserve(L, (size_t)S->maxBatch, tiles))) {
      fem_plan_destroy(plan);
      cudaFree(m.coords);
      cudaFree(m.states);
      cudaFree(m.residual);
      cudaFree(m.mat);
      S->used -= bytes;
      return st;
    }
  for (size_t i = 0; i < S->meshes.size(); i++)
    if (!S->meshes[i].plan) {
      S->meshes[i] = m;
      *meshId = (int)i;
      return FEM_SUCCESS;
    }
  S->meshes.push_back(m);
  *meshId = (int)S->meshes.size() - 1;
  return FEM_SUCCESS;
}

int fem_server_remove_mesh(fem_server *S, int meshId) {
  fem::clear_error();
  if (!S) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "server is NULL");
  ServerMesh m;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (meshId < 0 || meshId >= (int)S->meshes.size() || !S->meshes[meshId].plan)
      return fem::fail(FEM_ERR_INVALID_ARGUMENT, "no mesh %d", meshId);
    if (S->meshes[meshId].busy) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "mesh %d has a request in flight", meshId);
    m = S->meshes[meshId];
    S->meshes[meshId] = ServerMesh();
    S->used -= m.bytes;
  }
  cudaFree(m.coords);
  cudaFree(m.states);
  cudaFree(m.residual);
  cudaFree(m.mat);
  fem_plan_destroy(m.plan);
  return FEM_SUCCESS;
}

int fem_server_mesh_outputs(fem_server *S, int meshId, const double **residual, const double **matEntries,
                            const int **rowp, const int **cols, int64_t *nnzb) {
  fem::clear_error();
  if (!S) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "server is NULL");
  std::lock_guard<std::mutex> lk(S->mu);
  if (meshId < 0 || meshId >= (int)S->meshes.size() || !S->meshes[meshId].plan)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "no mesh %d", meshId);
  const ServerMesh &m = S->meshes[meshId];
  if (residual) *residual = m.residual;
  if (matEntries) *matEntries = m.mat;
  if (rowp) *rowp = m.plan->d_rowp;
  if (cols) *cols = m.plan->d_cols;
  if (nnzb) *nnzb = m.plan->nnzb;
  return FEM_SUCCESS;
}

int fem_server_submit(fem_server *S, int meshId, const double *hostStates, double *hostResidual, int64_t *ticket) {
  fem::clear_error();
  if (!S || !hostStates || !ticket) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  if (meshId < 0 || meshId >= (int)S->meshes.size() || !S->meshes[meshId].plan)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "no mesh %d", meshId);
  if (S->meshes[meshId].busy)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "mesh %d already has a request in flight", meshId);
  Request r;
  r.mesh = meshId;
  r.hostStates = hostStates;
  r.hostResidual = hostResidual;
  r.tSubmit = now_seconds();
  const int64_t tk = S->nextTicket++;
  S->reqs[tk] = r;
  S->meshes[meshId].busy = true;
  S->pending.push_back(tk);
  *ticket = tk;
  S->cvDispatch.notify_one();
  return FEM_SUCCESS;
}

int fem_server_wait(fem_server *S, int64_t ticket, int timeoutMs, double *latencySeconds) {
  fem::clear_error();
  if (!S) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "server is NULL");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "unknown ticket %lld", (long long)ticket);
  const bool ok = S->cvDone.wait_for(lk, std::chrono::milliseconds(timeoutMs < 0 ? 0 : timeoutMs),
                                     [&] { return S->reqs[ticket].done; });
  if (!ok) return fem::fail(FEM_ERR_UNSUPPORTED, "ticket %lld not finished after %d ms", (long long)ticket, timeoutMs);
  Request r = S->reqs[ticket];
  S->reqs.erase(ticket);
  if (latencySeconds) *latencySeconds = r.tDone - r.tSubmit;
  if (r.status) return fem::fail(r.status, "request %lld failed", (long long)ticket);
  return FEM_SUCCESS;
}

int fem_server_stats(fem_server *S, int64_t *waves, int64_t *completed, int64_t *elements, int64_t *usedBytes,
                     int64_t *budgetBytes) {
  fem::clear_error();
  if (!S) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "server is NULL");
  std::lock_guard<std::mutex> lk(S->mu);
  if (waves) *waves = S->waves;
  if (completed) *completed = S->completed;
  if (elements) *elements = S->elementsDone;
  if (usedBytes) *usedBytes = S->used;
  if (budgetBytes) *budgetBytes = S->budget;
  return FEM_SUCCESS;
}

}  // extern "C"
