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
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <string>
#include <vector>

#include "fem_common.h"
#include "fem_device.cuh"
#include "fem_launch.h"

namespace fem {
namespace dev {

// y = A x, 2x2 BSR, eight lanes per block row.
__global__ void __launch_bounds__(256) bsr_spmv_kernel(int numRows, const int *__restrict__ rowp,
                                                       const int *__restrict__ cols, const double *__restrict__ Av,
                                                       const double *__restrict__ x, double *__restrict__ y) {
  const int lane = threadIdx.x & 7;
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  if (row >= numRows) return;
  double y0 = 0, y1 = 0;
  const int b0 = __ldg(rowp + row), b1 = __ldg(rowp + row + 1);
  for (int j = b0 + lane; j < b1; j += 8) {
    const double2 *blk = reinterpret_cast<const double2 *>(Av) + 2 * (int64_t)j;
    const double2 r0 = __ldg(blk), r1 = __ldg(blk + 1);
    const double2 xv = __ldg(reinterpret_cast<const double2 *>(x) + __ldg(cols + j));
    y0 = fma(r0.x, xv.x, fma(r0.y, xv.y, y0));
    y1 = fma(r1.x, xv.x, fma(r1.y, xv.y, y1));
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    y0 += __shfl_down_sync(0xffffffffu, y0, o, 8);
    y1 += __shfl_down_sync(0xffffffffu, y1, o, 8);
  }
  if (lane == 0) reinterpret_cast<double2 *>(y)[row] = make_double2(y0, y1);
}

}  // namespace dev
}  // namespace fem

namespace fem {
namespace {
template <typename T>
int launch_any(int order, int mode, const dev::AsmArgs &a, cudaStream_t s) {
  using namespace dev;
  switch (mode) {
    case kRes: return launch_mode<T, kRes>(order, a, s);
    case kJac: return launch_mode<T, kJac>(order, a, s);
    case kRes | kJac: return launch_mode<T, kRes | kJac>(order, a, s);
    case kPlan | kRes: return launch_mode<T, kPlan | kRes>(order, a, s);
    case kPlan | kJac: return launch_mode<T, kPlan | kJac>(order, a, s);
    case kPlan | kRes | kJac: return launch_mode<T, kPlan | kRes | kJac>(order, a, s);
    default: return fail(FEM_ERR_INVALID_ARGUMENT, "bad kernel mode %d", mode);
  }
}
}  // namespace

// Order-4 MIXED element stiffness on the fifth-generation tensor cores (kU) when
// FEM_ORDER4_MIXED_STIFFNESS=tcgen05; the FP32 CUDA-core products otherwise, the
// faster form on B200 (2.63 against 3.44 ms for a 512^2 order-4 mesh: both forms
// are bound by the shared-memory side of the L1 data pipe, and the BF16 operand
// tiles and the staged accumulator add more of that traffic than the tensor cores
// take off the FMA pipe).
bool umma_order4() {
  static const bool on = [] {
    const char *v = std::getenv("FEM_ORDER4_MIXED_STIFFNESS");
    return v && std::string(v) == "tcgen05";
  }();
  return on;
}

int launch(int order, int precision, int mode, const dev::AsmArgs &a, cudaStream_t s, int strain) {
  if (strain == FEM_STRAIN_NONLINEAR) {
    if (precision != FEM_PRECISION_FP64)
      return fail(FEM_ERR_INVALID_ARGUMENT, "NONLINEAR strain is assembled in FP64 only (precision %d)", precision);
    if (frag_supported(order, precision, strain, (mode & dev::kPlan) != 0))
      return launch_frag(order, precision, mode, a, s, strain);
    return launch_nl(order, mode, a, s);
  }
  if (strain != FEM_STRAIN_LINEAR) return fail(FEM_ERR_INVALID_ARGUMENT, "strain type %d", strain);
  if ((mode & dev::kPlan) == 0 && frag_supported(order, precision, strain, false))
    return launch_frag(order, precision, mode, a, s);
  if (precision == FEM_PRECISION_FP64) return launch_any<double>(order, mode, a, s);
  if (precision == FEM_PRECISION_MIXED && order == 4 && (mode & dev::kJac) && umma_order4()) {
    using namespace dev;
    switch (mode) {
      case kJac: return launch_p<4, float, kJac | kU>(a, s);
      case kRes | kJac: return launch_p<4, float, kRes | kJac | kU>(a, s);
      case kPlan | kJac: return launch_p<4, float, kPlan | kJac | kU>(a, s);
      case kPlan | kRes | kJac: return launch_p<4, float, kPlan | kRes | kJac | kU>(a, s);
      default: return fail(FEM_ERR_INVALID_ARGUMENT, "bad kernel mode %d", mode);
    }
  }
  if (precision == FEM_PRECISION_MIXED) return launch_any<float>(order, mode, a, s);
  return fail(FEM_ERR_INVALID_ARGUMENT, "precision %d", precision);
}

namespace {
int run_dropin(int precision, bool jac, int order, const int *connPtr, const int *conn, int numElements,
               const double *states, const double *coords, double E, double nu, double t, const int *map,
               double *residual, double *mat, void *stream, double *elapsed, int strain = FEM_STRAIN_LINEAR) {
  clear_error();
  if (elapsed) *elapsed = 0.0;
  if (order < 1 || order > 4) return fail(FEM_ERR_INVALID_ORDER, "element order %d (supported: 1..4)", order);
  if (numElements < 0) return fail(FEM_ERR_INVALID_ARGUMENT, "numElements < 0");
  if (numElements == 0) return FEM_SUCCESS;
  if (!connPtr || !conn || !states || !coords) return fail(FEM_ERR_INVALID_ARGUMENT, "NULL input array");
  if (jac && (!map || !mat)) return fail(FEM_ERR_INVALID_ARGUMENT, "NULL map or matEntries");
  if (!jac && !residual) return fail(FEM_ERR_INVALID_ARGUMENT, "NULL residual");
  if (!aligned16(states) || !aligned16(coords) || (residual && !aligned16(residual)))
    return fail(FEM_ERR_MISALIGNED, "states, nodeCoords and residual must be 16-byte aligned");
  if (mat && (reinterpret_cast<uintptr_t>(mat) & 7u)) return fail(FEM_ERR_MISALIGNED, "matEntries not 8-byte aligned");
  dev::AsmArgs a{};
  a.connPtr = connPtr;
  a.conn = conn;
  a.map = map;
  a.states = states;
  a.coords = coords;
  a.residual = residual;
  a.mat = mat;
  a.begin = 0;
  a.count = numElements;
  set_material(a, E, nu, t);
  const int mode = (jac ? dev::kJac : 0) | (residual ? dev::kRes : 0);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return timed(s, elapsed, [&] { return launch(order, precision, mode, a, s, strain); });
}

}  // namespace
}  // namespace fem

// ---------------------------------------------------------------------------------------
// Plans
// ---------------------------------------------------------------------------------------

namespace {
void plan_free(fem_plan *p) {
  if (!p) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(p->device);
  cudaFree(p->d_rowp);
  cudaFree(p->d_cols);
  cudaFree(p->d_connList);
  cudaFree(p->d_blockCode);
  cudaFree(p->d_pairConnList);
  cudaFree(p->d_pairCode);
  cudaFree(p->d_rowElemPtr);
  cudaFree(p->d_rowElem);
  cudaFree(p->d_rowChunk);
  cudaFree(p->d_sched);
  cudaFree(p->d_waits);
  if (p->copyIn) cudaStreamDestroy(p->copyIn);
  if (p->copyOut) cudaStreamDestroy(p->copyOut);
  cudaSetDevice(cur);
  delete p;
}

template <typename V>
int upload(const std::vector<V> &h, V **d, int64_t &bytes) {
  const size_t n = h.size() * sizeof(V);
  cudaError_t err = cudaMalloc(reinterpret_cast<void **>(d), n ? n : 16);
  if (err != cudaSuccess) return fem::fail(FEM_ERR_CUDA, "cudaMalloc(%zu): %s", n, cudaGetErrorString(err));
  bytes += (int64_t)n;
  if (n) {
    err = cudaMemcpy(*d, h.data(), n, cudaMemcpyHostToDevice);
    if (err != cudaSuccess) return fem::fail(FEM_ERR_CUDA, "cudaMemcpy: %s", cudaGetErrorString(err));
  }
  return FEM_SUCCESS;
}
// Default band of the dependency-ordered schedule: about 8 MB of matrix blocks per
// band (one element row of the 1024^2 order-3 mesh), so that the few bands in
// flight between a band's first and last colour stay well inside the 126 MB L2.
int default_band(const fem_plan *p) {
  const double bytesPerElement = 32.0 * (double)p->nnzb / std::max(1, p->numElements);
  const double band = 8e6 / std::max(bytesPerElement, 1.0);
  return (int)std::min(65536.0, std::max(256.0, std::round(band / 2.0) * 2.0));
}

int default_tile(int order) { return order == 4 ? 8 : 16; }

// Builds the dependency-ordered schedule of `p`: bands of `band` consecutive element
// ids; group (k, c) = band k's elements of colour c, a list-position range (the
// list holds each colour's elements in ascending id).  Group (k, c) waits for, in
// every band k' whose node span [lowest, highest node id] meets band k's, the
// latest non-empty colour c' < c: any earlier-colour element sharing a node with
// band k's colour-c elements lies in such a band k', and its group is (k', c')
// or one that (k', c') waits for in turn.  Dispatch step t(k, c) = max(k, t of
// each dependency + 1); groups run in (t, c, k) order and are cut into tiles of
// `tile` list positions (even, so element pairs never straddle two tiles).
int build_schedule(fem_plan *p, int band, int tile) {
  cudaFree(p->d_sched);
  p->deviceBytes -= p->schedBytes;
  p->d_sched = nullptr;
  p->schedBytes = 0;
  p->schedBand = p->schedTile = p->schedGroups = p->schedTiles = 0;
  p->sched = fem::dev::SchedArgs{};
  if (band <= 0 || p->numElements == 0) return FEM_SUCCESS;
  const int nE = p->numElements, nc = p->numColours;
  band = std::max(2, band + (band & 1));
  tile = std::max(2, tile + (tile & 1));
  const int B = (int)(((int64_t)nE + band - 1) / band);
  if ((int64_t)B * nc > 4 * 1024 * 1024)
    return fem::fail(FEM_ERR_UNSUPPORTED, "schedule of %d bands x %d colours: use longer bands", B, nc);
  // per (band, colour): list positions; per band: node span
  std::vector<int64_t> p0((size_t)B * nc), p1((size_t)B * nc);
  std::vector<int> blo(B, INT32_MAX), bhi(B, -1);
  for (int c = 0; c < nc; c++) {
    const int *b0 = p->elemList.data() + p->colourPtr[c], *b1 = p->elemList.data() + p->colourPtr[c + 1];
    for (int k = 0; k < B; k++) {
      const size_t x = (size_t)k * nc + c;
      p0[x] = std::lower_bound(b0, b1, (int)((int64_t)k * band)) - p->elemList.data();
      p1[x] = std::lower_bound(b0, b1, (int)std::min<int64_t>((int64_t)(k + 1) * band, nE)) - p->elemList.data();
      for (int64_t q = p0[x]; q < p1[x]; q++) {
        blo[k] = std::min(blo[k], p->nodeLo[q]);
        bhi[k] = std::max(bhi[k], p->nodeHi[q]);
      }
    }
  }
  // bands whose node spans meet: sweep over bands ordered by span start
  std::vector<int> byLo(B);
  for (int k = 0; k < B; k++) byLo[k] = k;
  std::sort(byLo.begin(), byLo.end(), [&](int a, int b) { return blo[a] < blo[b]; });
  std::vector<std::vector<int>> meets(B);
  int64_t pairs = 0;
  for (int i = 0; i < B; i++) {
    const int k = byLo[i];
    if (bhi[k] < 0) continue;
    for (int j = i + 1; j < B && blo[byLo[j]] <= bhi[k]; j++) {
      const int k2 = byLo[j];
      if (bhi[k2] < 0) continue;
      meets[k].push_back(k2);
      meets[k2].push_back(k);
      if (++pairs > 64LL * B + 1024)
        return fem::fail(FEM_ERR_UNSUPPORTED, "band node spans overlap too widely for a schedule (scrambled numbering)");
    }
    meets[k].push_back(k);
  }
  // groups with their dependencies and steps
  struct Grp {
    int t, c, k;
    std::vector<int> deps;  // cell indices k * nc + c
  };
  std::vector<int> step((size_t)B * nc, -1);
  std::vector<Grp> gs;
  std::vector<int> cellGroup((size_t)B * nc, -1);
  for (int c = 0; c < nc; c++) {
    for (int k = 0; k < B; k++) {
      const size_t x = (size_t)k * nc + c;
      if (p1[x] <= p0[x]) continue;
      Grp g{k, c, k, {}};
      for (int k2 : meets[k]) {
        for (int c2 = c - 1; c2 >= 0; c2--) {
          const size_t y = (size_t)k2 * nc + c2;
          if (p1[y] > p0[y]) {
            g.deps.push_back((int)y);
            g.t = std::max(g.t, step[y] + 1);
            break;
          }
        }
      }
      step[x] = g.t;
      gs.push_back(std::move(g));
    }
  }
  std::vector<int> order(gs.size());
  for (size_t i = 0; i < gs.size(); i++) order[i] = (int)i;
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    const Grp &x = gs[a], &y = gs[b];
    return x.t != y.t ? x.t < y.t : (x.c != y.c ? x.c < y.c : x.k < y.k);
  });
  for (size_t i = 0; i < order.size(); i++) {
    const Grp &g = gs[order[i]];
    cellGroup[(size_t)g.k * nc + g.c] = (int)i;
  }
  const int G = (int)order.size();
  std::vector<fem::dev::SchedTile> tiles;
  std::vector<int> groupTiles(G), depPtr(G + 1, 0), deps;
  for (int i = 0; i < G; i++) {
    const Grp &g = gs[order[i]];
    const size_t x = (size_t)g.k * nc + g.c;
    int n = 0;
    for (int64_t q = p0[x]; q < p1[x]; q += tile, n++)
      tiles.push_back({q, (int)std::min<int64_t>(tile, p1[x] - q), i});
    groupTiles[i] = n;
    for (int y : g.deps) deps.push_back(cellGroup[y]);
    depPtr[i + 1] = (int)deps.size();
  }
  // one device allocation: tiles | groupTiles | depPtr | deps | status (2 + G words)
  auto al = [](size_t b) { return (b + 15) & ~(size_t)15; };
  const size_t oT = 0, oG = al(oT + tiles.size() * sizeof(fem::dev::SchedTile)), oP = al(oG + 4 * (size_t)G),
               oD = al(oP + 4 * (size_t)(G + 1)), oS = al(oD + 4 * std::max<size_t>(deps.size(), 1)),
               total = al(oS + 4 * (size_t)(G + 2));
  cudaError_t err = cudaMalloc(&p->d_sched, total);
  if (err != cudaSuccess) return fem::fail(FEM_ERR_CUDA, "cudaMalloc(%zu): %s", total, cudaGetErrorString(err));
  unsigned char *b = static_cast<unsigned char *>(p->d_sched);
  if ((err = cudaMemcpy(b + oT, tiles.data(), tiles.size() * sizeof(fem::dev::SchedTile), cudaMemcpyHostToDevice)) ||
      (err = cudaMemcpy(b + oG, groupTiles.data(), 4 * (size_t)G, cudaMemcpyHostToDevice)) ||
      (err = cudaMemcpy(b + oP, depPtr.data(), 4 * (size_t)(G + 1), cudaMemcpyHostToDevice)) ||
      (!deps.empty() && (err = cudaMemcpy(b + oD, deps.data(), 4 * deps.size(), cudaMemcpyHostToDevice))) ||
      (err = cudaMemset(b + oS, 0, 4 * (size_t)(G + 2)))) {
    cudaFree(p->d_sched);
    p->d_sched = nullptr;
    return fem::fail(FEM_ERR_CUDA, "schedule upload: %s", cudaGetErrorString(err));
  }
  if (int st = fem::uploads_visible("schedule upload")) {
    cudaFree(p->d_sched);
    p->d_sched = nullptr;
    return st;
  }
  p->schedBand = band;
  p->schedTile = tile;
  p->schedGroups = G;
  p->schedTiles = (int)tiles.size();
  p->schedBytes = (int64_t)total;
  p->deviceBytes += p->schedBytes;
  fem::dev::SchedArgs &a = p->sched;
  a.tiles = reinterpret_cast<const fem::dev::SchedTile *>(b + oT);
  a.groupTiles = reinterpret_cast<const int *>(b + oG);
  a.depPtr = reinterpret_cast<const int *>(b + oP);
  a.deps = reinterpret_cast<const int *>(b + oD);
  a.status = reinterpret_cast<int *>(b + oS);
  a.ntiles = p->schedTiles;
  a.stallGroup = -1;
  a.waitLimitNs = 500000000LL;
  return FEM_SUCCESS;
}

// Whether fem_plan_assemble runs `p` as one dependency-ordered launch.
bool plan_sched(const fem_plan *p, int precision, int strain) {
  return p->schedGroups > 0 && fem::frag_supported(p->order, precision, strain, true) &&
         !(fem::plan_rows(p) && strain == FEM_STRAIN_LINEAR);
}
}  // namespace

extern "C" {

int fem_run_residual(int elementOrder, const int *connPtr, const int *conn, int numElements, const double *states,
                     const double *nodeCoords, double E, double nu, double t, double *residual, void *stream,
                     double *elapsedSeconds) {
  return fem::run_dropin(FEM_PRECISION_FP64, false, elementOrder, connPtr, conn, numElements, states, nodeCoords, E,
                         nu, t, nullptr, residual, nullptr, stream, elapsedSeconds);
}

int fem_run_jacobian(int elementOrder, const int *connPtr, const int *conn, int numElements, const double *states,
                     const double *nodeCoords, double E, double nu, double t, const int *elementBCSRMap,
                     double *residual, double *matEntries, void *stream, double *elapsedSeconds) {
  return fem::run_dropin(FEM_PRECISION_FP64, true, elementOrder, connPtr, conn, numElements, states, nodeCoords, E,
                         nu, t, elementBCSRMap, residual, matEntries, stream, elapsedSeconds);
}

int fem_run_residual_mixed(int elementOrder, const int *connPtr, const int *conn, int numElements,
                           const double *states, const double *nodeCoords, double E, double nu, double t,
                           double *residual, void *stream, double *elapsedSeconds) {
  return fem::run_dropin(FEM_PRECISION_MIXED, false, elementOrder, connPtr, conn, numElements, states, nodeCoords, E,
                         nu, t, nullptr, residual, nullptr, stream, elapsedSeconds);
}

int fem_run_jacobian_mixed(int elementOrder, const int *connPtr, const int *conn, int numElements,
                           const double *states, const double *nodeCoords, double E, double nu, double t,
                           const int *elementBCSRMap, double *residual, double *matEntries, void *stream,
                           double *elapsedSeconds) {
  return fem::run_dropin(FEM_PRECISION_MIXED, true, elementOrder, connPtr, conn, numElements, states, nodeCoords, E,
                         nu, t, elementBCSRMap, residual, matEntries, stream, elapsedSeconds);
}

int fem_run_residual_ex(int elementOrder, const int *connPtr, const int *conn, int numElements, const double *states,
                        const double *nodeCoords, double E, double nu, double t, double *residual, int precision,
                        int strainType, void *stream, double *elapsedSeconds) {
  return fem::run_dropin(precision, false, elementOrder, connPtr, conn, numElements, states, nodeCoords, E, nu, t,
                         nullptr, residual, nullptr, stream, elapsedSeconds, strainType);
}

int fem_run_jacobian_ex(int elementOrder, const int *connPtr, const int *conn, int numElements, const double *states,
                        const double *nodeCoords, double E, double nu, double t, const int *elementBCSRMap,
                        double *residual, double *matEntries, int precision, int strainType, void *stream,
                        double *elapsedSeconds) {
  return fem::run_dropin(precision, true, elementOrder, connPtr, conn, numElements, states, nodeCoords, E, nu, t,
                         elementBCSRMap, residual, matEntries, stream, elapsedSeconds, strainType);
}

int fem_bsr_spmv(int numRows, const int *rowp, const int *cols, const double *A, const double *x, double *y,
                 void *stream) {
  fem::clear_error();
  if (numRows < 0) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "numRows < 0");
  if (numRows == 0) return FEM_SUCCESS;
  if (!rowp || !cols || !A || !x || !y) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL array");
  if (!fem::aligned16(A) || !fem::aligned16(x) || !fem::aligned16(y))
    return fem::fail(FEM_ERR_MISALIGNED, "A, x, y must be 16-byte aligned");
  const int64_t threads = (int64_t)numRows * 8;
  const int grid = (int)((threads + 255) / 256);
  fem::dev::bsr_spmv_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(numRows, rowp, cols, A, x, y);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return fem::cuda_fail(err, "bsr_spmv launch");
  return FEM_SUCCESS;
}

int fem_plan_create(int elementOrder, int numNodes, const int *connPtr, const int *conn, int numElements,
                    fem_plan **plan) {
  fem::clear_error();
  if (!plan) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan is NULL");
  *plan = nullptr;
  if (elementOrder < 1 || elementOrder > 4) return fem::fail(FEM_ERR_INVALID_ORDER, "element order %d", elementOrder);
  fem::HostPlan hp;
  int st = fem::build_host_plan(elementOrder, numNodes, connPtr, conn, numElements, hp);
  if (st) return st;
  fem_plan *p = new fem_plan();
  cudaGetDevice(&p->device);
  p->order = hp.order;
  p->nn = hp.nn;
  p->numNodes = hp.numNodes;
  p->numElements = hp.numElements;
  p->numColours = hp.numColours;
  p->nnzb = hp.nnzb;
  p->colourPtr = hp.colourPtr;
  p->elemList = hp.elemList;
  p->nodeLo.resize((size_t)hp.numElements);
  p->nodeHi.resize((size_t)hp.numElements);
  for (int k = 0; k < hp.numElements; k++) {
    const int *c = &hp.connList[(size_t)k * hp.nn];
    p->nodeLo[k] = *std::min_element(c, c + hp.nn);
    p->nodeHi[k] = *std::max_element(c, c + hp.nn);
  }
  if ((st = upload(std::vector<int>(1, 0), &p->d_waits, p->deviceBytes)) ||
      (st = upload(hp.rowp, &p->d_rowp, p->deviceBytes)) || (st = upload(hp.cols, &p->d_cols, p->deviceBytes)) ||
      (st = upload(hp.connList, &p->d_connList, p->deviceBytes)) ||
      (st = upload(hp.blockCode, &p->d_blockCode, p->deviceBytes))) {
    plan_free(p);
    return st;
  }
  if (!hp.rowChunk.empty()) {
    if ((st = upload(hp.rowElemPtr, &p->d_rowElemPtr, p->deviceBytes)) ||
        (st = upload(hp.rowElem, &p->d_rowElem, p->deviceBytes)) ||
        (st = upload(hp.rowChunk, &p->d_rowChunk, p->deviceBytes))) {
      plan_free(p);
      return st;
    }
    p->numChunks = (int)hp.rowChunk.size() - 1;
  }
  if (hp.numPairColours > 0) {
    if ((st = upload(hp.pairConnList, &p->d_pairConnList, p->deviceBytes)) ||
        (st = upload(hp.pairCode, &p->d_pairCode, p->deviceBytes))) {
      plan_free(p);
      return st;
    }
    p->pairColourPtr = hp.pairColourPtr;
    p->pairRegionEnd = hp.pairRegionEnd;
    p->pairList = hp.pairList;
    p->pairNodeLo.resize((size_t)hp.numElements);
    p->pairNodeHi.resize((size_t)hp.numElements);
    for (int k = 0; k < hp.numElements; k++) {
      const int *c = &hp.pairConnList[(size_t)k * hp.nn];
      p->pairNodeLo[k] = *std::min_element(c, c + hp.nn);
      p->pairNodeHi[k] = *std::max_element(c, c + hp.nn);
    }
    p->numPairColours = hp.numPairColours;
    p->numPairs = hp.numPairs;
    p->usePairs = true;
  }
  if ((st = fem::uploads_visible("fem_plan_create: table upload"))) {
    plan_free(p);
    return st;
  }
  *plan = p;
  return FEM_SUCCESS;
}

int fem_plan_set_schedule(fem_plan *plan, int bandElements, int tileElements) {
  fem::clear_error();
  if (!plan) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (plan->order < 2) return fem::fail(FEM_ERR_UNSUPPORTED, "order-1 plans assemble by rows (or colours)");
  if (bandElements < -1 || tileElements < 0) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "bad band or tile length");
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(plan->device);
  const int st = build_schedule(plan, bandElements < 0 ? default_band(plan) : bandElements,
                                tileElements ? tileElements : default_tile(plan->order));
  cudaSetDevice(cur);
  return st;
}

int fem_plan_get_schedule(const fem_plan *plan, int *bandElements, int *tileElements, int *numGroups, int *numTiles) {
  fem::clear_error();
  if (!plan) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (bandElements) *bandElements = plan->schedBand;
  if (tileElements) *tileElements = plan->schedTile;
  if (numGroups) *numGroups = plan->schedGroups;
  if (numTiles) *numTiles = plan->schedTiles;
  return FEM_SUCCESS;
}

int fem_plan_get_schedule_tables(const fem_plan *plan, int64_t *tileBegin, int *tileCount, int *tileGroup,
                                 int *groupTiles, int *depPtr, int *deps) {
  fem::clear_error();
  if (!plan) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (!plan->d_sched) return FEM_SUCCESS;
  const fem::dev::SchedArgs &a = plan->sched;
  const int G = plan->schedGroups, T = plan->schedTiles;
  std::vector<fem::dev::SchedTile> t((size_t)T);
  std::vector<int> ptr((size_t)G + 1);
  cudaError_t err = cudaMemcpy(t.data(), a.tiles, sizeof(fem::dev::SchedTile) * (size_t)T, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess) err = cudaMemcpy(ptr.data(), a.depPtr, sizeof(int) * ((size_t)G + 1), cudaMemcpyDeviceToHost);
  if (err == cudaSuccess && groupTiles)
    err = cudaMemcpy(groupTiles, a.groupTiles, sizeof(int) * (size_t)G, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess && deps && ptr[G] > 0)
    err = cudaMemcpy(deps, a.deps, sizeof(int) * (size_t)ptr[G], cudaMemcpyDeviceToHost);
  if (err != cudaSuccess) return fem::cuda_fail(err, "cudaMemcpy(schedule tables)");
  for (int i = 0; i < T; i++) {
    if (tileBegin) tileBegin[i] = t[i].begin;
    if (tileCount) tileCount[i] = t[i].count;
    if (tileGroup) tileGroup[i] = t[i].group;
  }
  if (depPtr) std::copy(ptr.begin(), ptr.end(), depPtr);
  return FEM_SUCCESS;
}

int fem_plan_wait_status(fem_plan *plan, void *stream, int64_t *timedOutWaits) {
  fem::clear_error();
  if (!plan || !timedOutWaits) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  *timedOutWaits = 0;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int v[2] = {0, 0};
  cudaError_t err = cudaMemcpyAsync(&v[0], plan->d_waits, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess && plan->d_sched)
    err = cudaMemcpyAsync(&v[1], plan->sched.status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err == cudaSuccess && v[0]) err = cudaMemsetAsync(plan->d_waits, 0, sizeof(int), s);
  if (err == cudaSuccess && v[1]) err = cudaMemsetAsync(plan->sched.status, 0, sizeof(int), s);
  if (err == cudaSuccess && (v[0] || v[1])) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return fem::cuda_fail(err, "reading the wait status");
  *timedOutWaits = (int64_t)v[0] + v[1];
  return FEM_SUCCESS;
}

int fem_plan_set_schedule_waits(fem_plan *plan, int64_t waitLimitNs, int stallGroup) {
  fem::clear_error();
  if (!plan) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (stallGroup != -1 && (stallGroup < 0 || stallGroup >= plan->schedGroups))
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "stallGroup %d of %d groups", stallGroup, plan->schedGroups);
  if (waitLimitNs > 0) plan->sched.waitLimitNs = waitLimitNs;
  plan->sched.stallGroup = stallGroup;
  return FEM_SUCCESS;
}

int fem_plan_destroy(fem_plan *plan) {
  fem::clear_error();
  plan_free(plan);
  return FEM_SUCCESS;
}

int fem_plan_info(const fem_plan *plan, int *numNodes, int *numElements, int64_t *nnzb, int *numColours,
                  int64_t *deviceBytes) {
  fem::clear_error();
  if (!plan) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (numNodes) *numNodes = plan->numNodes;
  if (numElements) *numElements = plan->numElements;
  if (nnzb) *nnzb = plan->nnzb;
  if (numColours) *numColours = plan->numColours;
  if (deviceBytes) *deviceBytes = plan->deviceBytes;
  return FEM_SUCCESS;
}

int fem_plan_row_chunks(const fem_plan *plan, int *numChunks) {
  fem::clear_error();
  if (!plan || !numChunks) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  *numChunks = plan->numChunks;
  return FEM_SUCCESS;
}

int fem_plan_get_pattern(const fem_plan *plan, int *rowp, int *cols) {
  fem::clear_error();
  if (!plan || !rowp || !cols) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL argument");
  cudaError_t err = cudaMemcpy(rowp, plan->d_rowp, sizeof(int) * ((size_t)plan->numNodes + 1), cudaMemcpyDeviceToHost);
  if (err == cudaSuccess) err = cudaMemcpy(cols, plan->d_cols, sizeof(int) * (size_t)plan->nnzb, cudaMemcpyDeviceToHost);
  if (err != cudaSuccess) return fem::cuda_fail(err, "cudaMemcpy");
  return FEM_SUCCESS;
}

int fem_plan_device_pattern(const fem_plan *plan, const int **rowp, const int **cols) {
  fem::clear_error();
  if (!plan) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (rowp) *rowp = plan->d_rowp;
  if (cols) *cols = plan->d_cols;
  return FEM_SUCCESS;
}

int fem_plan_assemble(const fem_plan *plan, const double *states, const double *nodeCoords, double E, double nu,
                      double t, double *residual, double *matEntries, int precision, void *stream,
                      double *elapsedSeconds) {
  return fem_plan_assemble_ex(plan, states, nodeCoords, E, nu, t, residual, matEntries, precision, FEM_STRAIN_LINEAR,
                              stream, elapsedSeconds);
}

int fem_plan_assemble_ex(const fem_plan *plan, const double *states, const double *nodeCoords, double E, double nu,
                         double t, double *residual, double *matEntries, int precision, int strainType, void *stream,
                         double *elapsedSeconds) {
  fem::clear_error();
  if (elapsedSeconds) *elapsedSeconds = 0.0;
  if (!plan) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (!states || !nodeCoords) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL input array");
  if (!residual && !matEntries) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "no output requested");
  if (!fem::aligned16(states) || !fem::aligned16(nodeCoords) || (residual && !fem::aligned16(residual)))
    return fem::fail(FEM_ERR_MISALIGNED, "states, nodeCoords and residual must be 16-byte aligned");
  if (matEntries && (reinterpret_cast<uintptr_t>(matEntries) & 31u))
    return fem::fail(FEM_ERR_MISALIGNED, "matEntries must be 32-byte aligned (one 2x2 block per 256-bit store)");
  if (plan->numElements == 0) return FEM_SUCCESS;
  fem::dev::AsmArgs a{};
  fem::plan_args(a, plan);
  a.states = states;
  a.coords = nodeCoords;
  a.residual = residual;
  a.mat = matEntries;
  fem::set_material(a, E, nu, t);
  const int mode = fem::dev::kPlan | (residual ? fem::dev::kRes : 0) | (matEntries ? fem::dev::kJac : 0);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (fem::plan_rows(plan) && strainType == FEM_STRAIN_LINEAR) {
    // order 1: row assembly (FP64 arithmetic for both precisions)
    if (precision != FEM_PRECISION_FP64 && precision != FEM_PRECISION_MIXED)
      return fem::fail(FEM_ERR_INVALID_ARGUMENT, "precision %d", precision);
    a.begin = 0;
    a.count = plan->numChunks;
    return fem::timed(s, elapsedSeconds, [&] { return fem::launch_rows(mode, a, s); });
  }
  const bool frag = fem::frag_supported(plan->order, precision, strainType, true);
  if (plan_sched(plan, precision, strainType)) {
    // all colours in one dependency-ordered launch; the tile dispenser and the
    // per-group counters start at zero, the sticky timeout count (word 0) is kept
    const int st = fem::timed(s, elapsedSeconds, [&]() -> int {
      cudaError_t err = cudaMemsetAsync(plan->sched.status + 1, 0, sizeof(int) * ((size_t)plan->schedGroups + 1), s);
      if (err != cudaSuccess) return fem::cuda_fail(err, "cudaMemsetAsync(schedule counters)");
      return fem::launch_frag_sched(plan->order, precision, mode, a, plan->sched, s, strainType);
    });
    if (st || !elapsedSeconds) return st;
    int64_t waits = 0;
    const int st2 = fem_plan_wait_status(const_cast<fem_plan *>(plan), stream, &waits);
    if (st2) return st2;
    if (waits) return fem::fail(FEM_ERR_TIMEOUT, "%lld in-kernel waits of the dependency-ordered launch ran out",
                                (long long)waits);
    return st;
  }
  // the fragment kernel runs the pair layout (a step's two elements share an edge,
  // so the lines of the rows they share are written while they are still in L2)
  const bool pairs = frag && plan->usePairs && plan->numPairColours > 0;
  if (pairs) {
    a.connList = plan->d_pairConnList;
    a.blockCode = plan->d_pairCode;
  }
  const std::vector<int> &cptr = pairs ? plan->pairColourPtr : plan->colourPtr;
  const int ncol = pairs ? plan->numPairColours : plan->numColours;
  return fem::timed(s, elapsedSeconds, [&] {
    for (int c = 0; c < ncol; c++) {
      a.begin = cptr[c];
      a.count = cptr[c + 1] - cptr[c];
      int st = frag ? fem::launch_frag(plan->order, precision, mode, a, s, strainType, /*chained=*/c > 0)
                    : fem::launch(plan->order, precision, mode, a, s, strainType);
      if (st) return st;
    }
    return (int)FEM_SUCCESS;
  });
}

int fem_plan_set_layout(fem_plan *plan, int layout) {
  fem::clear_error();
  if (!plan) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (layout != FEM_LAYOUT_COLOURS && layout != FEM_LAYOUT_PAIRS)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "layout %d", layout);
  if (layout == FEM_LAYOUT_PAIRS && plan->numPairColours == 0)
    return fem::fail(FEM_ERR_UNSUPPORTED, "this plan has no pair layout (order 1, or its pairs need > 64 colours)");
  plan->usePairs = layout == FEM_LAYOUT_PAIRS;
  return FEM_SUCCESS;
}

int fem_plan_get_layout(const fem_plan *plan, int *layout, int64_t *numPairs, int *numPairColours) {
  fem::clear_error();
  if (!plan) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (layout) *layout = plan->usePairs ? FEM_LAYOUT_PAIRS : FEM_LAYOUT_COLOURS;
  if (numPairs) *numPairs = plan->numPairs;
  if (numPairColours) *numPairColours = plan->numPairColours;
  return FEM_SUCCESS;
}

// Host-buffer assembly with the copies overlapped: see include/fem_b200.h.  The
// schedule cuts the elements into bands (element-id ranges) and the nodes into as
// many chunks; launch (band k, colour c) runs after every launch (k', c - 1) whose
// band's node span overlaps band k's (t(k, c) = max(k, t(k', c - 1) + 1)), so every
// block still receives its colours in order and the result equals
// fem_plan_assemble's bit for bit.
int fem_plan_assemble_host(const fem_plan *plan, const double *hostStates, double *states, const double *nodeCoords,
                           double E, double nu, double t, double *hostResidual, double *residual, double *matEntries,
                           int precision, int strainType, int numBands, void *stream, double *elapsedSeconds) {
  fem::clear_error();
  if (elapsedSeconds) *elapsedSeconds = 0.0;
  if (!plan) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (!hostStates || !states || !nodeCoords || !hostResidual || !residual)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL state, coordinate or residual array");
  if (numBands < 1 || numBands > 256) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "numBands %d (1..256)", numBands);
  if (!fem::aligned16(states) || !fem::aligned16(nodeCoords) || !fem::aligned16(residual))
    return fem::fail(FEM_ERR_MISALIGNED, "states, nodeCoords and residual must be 16-byte aligned");
  if (matEntries && (reinterpret_cast<uintptr_t>(matEntries) & 31u))
    return fem::fail(FEM_ERR_MISALIGNED, "matEntries must be 32-byte aligned (one 2x2 block per 256-bit store)");
  if (strainType != FEM_STRAIN_LINEAR && strainType != FEM_STRAIN_NONLINEAR)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "strain type %d", strainType);
  if (precision != FEM_PRECISION_FP64 && precision != FEM_PRECISION_MIXED)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "precision %d", precision);
  if (strainType == FEM_STRAIN_NONLINEAR && precision != FEM_PRECISION_FP64)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NONLINEAR strain is assembled in FP64 only (precision %d)", precision);
  if (plan->numElements == 0) return FEM_SUCCESS;
  fem_plan *mp = const_cast<fem_plan *>(plan);  // the copy streams are created on first use
  for (cudaStream_t *cs : {&mp->copyIn, &mp->copyOut}) {
    if (!*cs) {
      cudaError_t err = cudaStreamCreateWithFlags(cs, cudaStreamNonBlocking);
      if (err != cudaSuccess) return fem::cuda_fail(err, "cudaStreamCreateWithFlags");
    }
  }
  const bool frag = fem::frag_supported(plan->order, precision, strainType, true);
  const bool rows = fem::plan_rows(plan) && strainType == FEM_STRAIN_LINEAR;
  // the fragment kernel runs the pair layout when the plan uses it (each band's pairs
  // and unpaired elements are two ranges of a colour), else the colour layout
  const bool pairs = frag && !rows && plan->usePairs && plan->numPairColours > 0;
  const int N = plan->numNodes, nE = plan->numElements;
  const int nc = pairs ? plan->numPairColours : plan->numColours;
  const std::vector<int> &cptr = pairs ? plan->pairColourPtr : plan->colourPtr;
  const std::vector<int> &list = pairs ? plan->pairList : plan->elemList;
  const std::vector<int> &nlo = pairs ? plan->pairNodeLo : plan->nodeLo;
  const std::vector<int> &nhi = pairs ? plan->pairNodeHi : plan->nodeHi;
  const int B = std::min(numBands, std::max(1, std::min(N, nE)));
  // node chunk j = [nstart[j], nstart[j + 1]); chunk_of inverts exactly that split
  std::vector<int64_t> nstart((size_t)B + 1);
  for (int j = 0; j <= B; j++) nstart[j] = (int64_t)j * N / B;
  auto chunk_of = [&](int64_t n) {
    return (int)(std::upper_bound(nstart.begin(), nstart.end(), n) - nstart.begin()) - 1;
  };
  auto node0 = [&](int j) { return nstart[j]; };

  // a (band, colour) cell: list positions [p0, p1) and, in the pair layout, the
  // band's unpaired elements [q0, q1)
  struct L {
    int t, c, k;
    int64_t p0, p1, q0, q1;
    int lo, hi;
  };
  std::vector<L> ls;
  if (rows) {
    ls.push_back({0, 0, 0, 0, plan->numChunks, 0, 0, 0, N - 1});
  } else {
    // per (band, colour): list positions and node span; per band: node span
    std::vector<int> blo(B, INT32_MAX), bhi(B, -1);
    std::vector<L> cells((size_t)B * nc);
    for (int c = 0; c < nc; c++) {
      // colour layout: the colour's elements in ascending id; pair layout: its pairs
      // in ascending id of their first element (two positions each), then its
      // unpaired elements in ascending id
      const int64_t c0 = cptr[c], c1 = cptr[c + 1], pe = pairs ? plan->pairRegionEnd[c] : c1;
      auto pair_pos = [&](int id) {  // first pair position whose lead id is >= id
        int64_t lo = 0, hi = (pe - c0) / 2;
        while (lo < hi) {
          const int64_t mid = (lo + hi) / 2;
          if (list[c0 + 2 * mid] < id) lo = mid + 1;
          else hi = mid;
        }
        return c0 + 2 * lo;
      };
      const int *s0 = list.data() + pe, *s1 = list.data() + c1;
      for (int k = 0; k < B; k++) {
        L &x = cells[(size_t)k * nc + c];
        x.c = c;
        x.k = k;
        const int id0 = (int)((int64_t)k * nE / B), id1 = (int)((int64_t)(k + 1) * nE / B);
        if (pairs) {
          x.p0 = pair_pos(id0);
          x.p1 = pair_pos(id1);
          x.q0 = std::lower_bound(s0, s1, id0) - list.data();
          x.q1 = std::lower_bound(s0, s1, id1) - list.data();
        } else {
          x.p0 = std::lower_bound(list.data() + c0, list.data() + c1, id0) - list.data();
          x.p1 = std::lower_bound(list.data() + c0, list.data() + c1, id1) - list.data();
          x.q0 = x.q1 = 0;
        }
        x.lo = INT32_MAX;
        x.hi = -1;
        for (int64_t q = x.p0; q < x.p1; q++) {
          x.lo = std::min(x.lo, nlo[q]);
          x.hi = std::max(x.hi, nhi[q]);
        }
        for (int64_t q = x.q0; q < x.q1; q++) {
          x.lo = std::min(x.lo, nlo[q]);
          x.hi = std::max(x.hi, nhi[q]);
        }
        blo[k] = std::min(blo[k], x.lo);
        bhi[k] = std::max(bhi[k], x.hi);
      }
    }
    std::vector<int> tprev(B), tcur(B);
    for (int k = 0; k < B; k++) tprev[k] = k;
    for (int c = 0; c < nc; c++) {
      for (int k = 0; k < B; k++) {
        int tk = k;
        if (c > 0)
          for (int k2 = 0; k2 < B; k2++)
            if (bhi[k2] >= 0 && bhi[k] >= 0 && blo[k2] <= bhi[k] && blo[k] <= bhi[k2]) tk = std::max(tk, tprev[k2] + 1);
        tcur[k] = tk;
        L &x = cells[(size_t)k * nc + c];
        x.t = tk;
        if (x.p1 > x.p0 || x.q1 > x.q0) ls.push_back(x);
      }
      tprev = tcur;
    }
    std::sort(ls.begin(), ls.end(), [](const L &a, const L &b) {
      return a.t != b.t ? a.t < b.t : (a.c != b.c ? a.c < b.c : a.k < b.k);
    });
  }
  // launches: the fragment kernel takes the ranges of one schedule step (independent:
  // different bands of different colours, or one colour's bands) in one launch
  struct G {
    int need, lo, hi;
    fem::dev::RangeList r;
  };
  std::vector<G> gs;
  for (const L &x : ls) {
    const int nr = (x.p1 > x.p0) + (x.q1 > x.q0);
    const bool join = frag && !rows && !gs.empty() && gs.back().r.n + nr <= fem::dev::kMaxRanges &&
                      ls[&x - ls.data() - 1].t == x.t;
    if (!join) gs.push_back(G{-1, INT32_MAX, -1, fem::dev::RangeList{0, {}, {}}});
    G &g = gs.back();
    for (int h = 0; h < 2; h++) {
      const int64_t b0 = h ? x.q0 : x.p0, b1 = h ? x.q1 : x.p1;
      if (b1 <= b0) continue;
      g.r.begin[g.r.n] = b0;
      g.r.count[g.r.n] = b1 - b0;
      g.r.n++;
    }
    g.lo = std::min(g.lo, x.lo);
    g.hi = std::max(g.hi, x.hi);
    g.need = rows ? B - 1 : std::max(g.need, chunk_of(x.hi));
  }
  // the last launch touching each node chunk (-1: none)
  std::vector<int> last(B, -1);
  for (int i = 0; i < (int)gs.size(); i++)
    for (int j = chunk_of(gs[i].lo); j <= chunk_of(gs[i].hi); j++) last[j] = i;

  fem::dev::AsmArgs a{};
  fem::plan_args(a, plan);
  if (pairs) {
    a.connList = plan->d_pairConnList;
    a.blockCode = plan->d_pairCode;
  }
  a.states = states;
  a.coords = nodeCoords;
  a.residual = residual;
  a.mat = matEntries;
  fem::set_material(a, E, nu, t);
  const int mode = fem::dev::kPlan | fem::dev::kRes | (matEntries ? fem::dev::kJac : 0);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  std::vector<cudaEvent_t> evs;
  auto event = [&](cudaEvent_t *e) {
    cudaError_t err = cudaEventCreateWithFlags(e, cudaEventDisableTiming);
    if (err == cudaSuccess) evs.push_back(*e);
    return err;
  };
  const int st = fem::timed(s, elapsedSeconds, [&]() -> int {
    cudaError_t err;
    cudaEvent_t start;
    if ((err = event(&start)) != cudaSuccess || (err = cudaEventRecord(start, s)) != cudaSuccess ||
        (err = cudaStreamWaitEvent(mp->copyIn, start, 0)) != cudaSuccess ||
        (err = cudaStreamWaitEvent(mp->copyOut, start, 0)) != cudaSuccess)
      return fem::cuda_fail(err, "stream ordering");
    std::vector<cudaEvent_t> in(B), done(gs.size(), nullptr);
    for (int j = 0; j < B; j++) {
      const int64_t n0 = node0(j), n1 = node0(j + 1);
      if (n1 > n0 && (err = cudaMemcpyAsync(states + 2 * n0, hostStates + 2 * n0, 16 * (size_t)(n1 - n0),
                                            cudaMemcpyHostToDevice, mp->copyIn)) != cudaSuccess)
        return fem::cuda_fail(err, "state upload");
      if ((err = event(&in[j])) != cudaSuccess || (err = cudaEventRecord(in[j], mp->copyIn)) != cudaSuccess)
        return fem::cuda_fail(err, "cudaEventRecord");
    }
    int waited = -1;
    for (int i = 0; i < (int)gs.size(); i++) {
      const G &g = gs[i];
      if (g.need > waited) {
        if ((err = cudaStreamWaitEvent(s, in[g.need], 0)) != cudaSuccess)
          return fem::cuda_fail(err, "cudaStreamWaitEvent");
        waited = g.need;
      }
      int r;
      if (rows) {
        a.begin = 0;
        a.count = plan->numChunks;
        r = fem::launch_rows(mode, a, s);
      } else if (frag) {
        // after the first launch each one follows this call's previous launch (a state
        // chunk it waits for still gates it through the stream's event wait)
        r = fem::launch_frag_ranges(plan->order, precision, mode, a, g.r, s, strainType, /*chained=*/i > 0);
      } else {
        a.begin = g.r.begin[0];
        a.count = g.r.count[0];
        r = fem::launch(plan->order, precision, mode, a, s, strainType);
      }
      if (r) return r;
      if (std::find(last.begin(), last.end(), i) != last.end()) {
        if ((err = event(&done[i])) != cudaSuccess || (err = cudaEventRecord(done[i], s)) != cudaSuccess)
          return fem::cuda_fail(err, "cudaEventRecord");
      }
    }
    // residual chunks, each once the last launch touching its nodes has run
    std::vector<int> order(B);
    for (int j = 0; j < B; j++) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return last[x] < last[y]; });
    for (int j : order) {
      const int64_t n0 = node0(j), n1 = node0(j + 1);
      if (n1 <= n0) continue;
      if (last[j] >= 0 && (err = cudaStreamWaitEvent(mp->copyOut, done[last[j]], 0)) != cudaSuccess)
        return fem::cuda_fail(err, "cudaStreamWaitEvent");
      if ((err = cudaMemcpyAsync(hostResidual + 2 * n0, residual + 2 * n0, 16 * (size_t)(n1 - n0),
                                 cudaMemcpyDeviceToHost, mp->copyOut)) != cudaSuccess)
        return fem::cuda_fail(err, "residual download");
    }
    cudaEvent_t end;
    if ((err = event(&end)) != cudaSuccess || (err = cudaEventRecord(end, mp->copyOut)) != cudaSuccess ||
        (err = cudaStreamWaitEvent(s, end, 0)) != cudaSuccess ||
        (err = cudaStreamWaitEvent(s, in[B - 1], 0)) != cudaSuccess)
      return fem::cuda_fail(err, "stream ordering");
    return (int)FEM_SUCCESS;
  });
  for (cudaEvent_t e : evs) cudaEventDestroy(e);
  return st;
}

}  // extern "C"
