// Host-side topology work of libfemb200: BSR pattern, element -> block map,
// element colouring and the compact per-element block codes of an assembly
// plan.  All integer work, exact and deterministic (OpenMP only where the
// result does not depend on the schedule).
#include <algorithm>
#include <climits>
#include <cstdarg>
#include <cstring>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "fem_common.h"

namespace fem {

namespace {
thread_local std::string g_last_error;

int validate_mesh(int numNodes, const int *connPtr, const int *conn, int numElements) {
  if (numNodes < 0 || numElements < 0) return fail(FEM_ERR_INVALID_ARGUMENT, "negative size");
  if (numElements > 0 && (!connPtr || !conn)) return fail(FEM_ERR_INVALID_ARGUMENT, "connPtr/conn is NULL");
  for (int e = 0; e < numElements; e++)
    if (connPtr[e + 1] < connPtr[e]) return fail(FEM_ERR_INVALID_ARGUMENT, "connPtr decreases at element %d", e);
  const int64_t total = numElements > 0 ? (int64_t)connPtr[numElements] : 0;
  int64_t bad = -1;
#pragma omp parallel for reduction(max : bad)
  for (int64_t i = numElements > 0 ? connPtr[0] : 0; i < total; i++)
    if (conn[i] < 0 || conn[i] >= numNodes) bad = std::max(bad, i);
  if (bad >= 0) return fail(FEM_ERR_INVALID_ARGUMENT, "conn[%lld] = %d outside [0, %d)", (long long)bad, conn[bad], numNodes);
  return FEM_SUCCESS;
}

// node -> incident elements (CSR), counting sort in element order.
void node_elements(int numNodes, const int *connPtr, const int *conn, int numElements, std::vector<int64_t> &ptr,
                   std::vector<int> &elems) {
  ptr.assign((size_t)numNodes + 1, 0);
  for (int e = 0; e < numElements; e++)
    for (int i = connPtr[e]; i < connPtr[e + 1]; i++) ptr[(size_t)conn[i] + 1]++;
  for (int r = 0; r < numNodes; r++) ptr[r + 1] += ptr[r];
  elems.resize((size_t)ptr[numNodes]);
  std::vector<int64_t> fill(ptr.begin(), ptr.end() - 1);
  for (int e = 0; e < numElements; e++)
    for (int i = connPtr[e]; i < connPtr[e + 1]; i++) elems[(size_t)fill[conn[i]]++] = e;
}

// Sorted unique neighbours of node r into buf.
inline void row_neighbours(int r, const std::vector<int64_t> &nptr, const std::vector<int> &nelem,
                           const int *connPtr, const int *conn, std::vector<int> &buf) {
  buf.clear();
  for (int64_t k = nptr[r]; k < nptr[r + 1]; k++) {
    const int e = nelem[(size_t)k];
    buf.insert(buf.end(), conn + connPtr[e], conn + connPtr[e + 1]);
  }
  std::sort(buf.begin(), buf.end());
  buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
}
}  // namespace

int fail(int status, const char *fmt, ...) {
  char msg[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof msg, fmt, ap);
  va_end(ap);
  g_last_error = msg;
  return status;
}

void clear_error() { g_last_error.clear(); }

const char *last_error_cstr() { return g_last_error.c_str(); }

int build_pattern(int numNodes, const int *connPtr, const int *conn, int numElements, int *rowp, int *cols,
                  int64_t *nnzb) {
  if (!rowp && !nnzb) return fail(FEM_ERR_INVALID_ARGUMENT, "rowp and nnzb are both NULL");
  int st = validate_mesh(numNodes, connPtr, conn, numElements);
  if (st) return st;
  std::vector<int64_t> nptr;
  std::vector<int> nelem;
  node_elements(numNodes, connPtr, conn, numElements, nptr, nelem);
  std::vector<int64_t> len((size_t)numNodes + 1, 0);
#pragma omp parallel
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 1024)
    for (int r = 0; r < numNodes; r++) {
      row_neighbours(r, nptr, nelem, connPtr, conn, buf);
      len[(size_t)r + 1] = (int64_t)buf.size();
    }
  }
  for (int r = 0; r < numNodes; r++) len[r + 1] += len[r];
  const int64_t total = len[numNodes];
  if (nnzb) *nnzb = total;
  if (total > INT_MAX) return fail(FEM_ERR_OVERFLOW, "nnzb = %lld does not fit int32 row pointers", (long long)total);
  if (rowp)
    for (int r = 0; r <= numNodes; r++) rowp[r] = (int)len[r];
  if (cols) {
#pragma omp parallel
    {
      std::vector<int> buf;
#pragma omp for schedule(dynamic, 1024)
      for (int r = 0; r < numNodes; r++) {
        row_neighbours(r, nptr, nelem, connPtr, conn, buf);
        std::copy(buf.begin(), buf.end(), cols + len[r]);
      }
    }
  }
  return FEM_SUCCESS;
}

int colour_greedy(int numNodes, const int *connPtr, const int *conn, int numElements, int *colour,
                  int *numColours) {
  if (!colour || !numColours) return fail(FEM_ERR_INVALID_ARGUMENT, "colour/numColours is NULL");
  int st = validate_mesh(numNodes, connPtr, conn, numElements);
  if (st) return st;
  std::vector<uint64_t> used((size_t)numNodes, 0);
  int nc = 0;
  for (int e = 0; e < numElements; e++) {
    uint64_t m = 0;
    for (int i = connPtr[e]; i < connPtr[e + 1]; i++) m |= used[conn[i]];
    if (~m == 0) return fail(FEM_ERR_UNSUPPORTED, "element %d needs more than 64 colours", e);
    const int c = __builtin_ctzll(~m);
    colour[e] = c;
    nc = std::max(nc, c + 1);
    for (int i = connPtr[e]; i < connPtr[e + 1]; i++) used[conn[i]] |= (1ull << c);
  }
  *numColours = nc;
  return FEM_SUCCESS;
}

// Row assembly tables of an order-1 plan (see HostPlan).  Left empty (the plan then
// assembles by colours) when a row is longer than one chunk or the element count
// does not fit the k << 2 packing.
static void build_row_plan(HostPlan &hp) {
  const int N = hp.numNodes, nE = hp.numElements;
  if (nE >= (1 << 29)) return;
  for (int r = 0; r < N; r++)
    if (hp.rowp[r + 1] - hp.rowp[r] > kRowChunkBlocks) return;
  std::vector<int> ptr((size_t)N + 1, 0);
  for (int64_t i = 0; i < (int64_t)nE * 4; i++) ptr[hp.connList[i] + 1]++;
  for (int r = 0; r < N; r++) ptr[r + 1] += ptr[r];
  std::vector<int> ent((size_t)ptr[N] * 2);
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int k = 0; k < nE; k++) {  // ascending k: each row lists its elements in colour order
    const uint8_t *rec = &hp.blockCode[(size_t)k * hp.codeStride];
    for (int a = 0; a < 4; a++) {
      const int r = hp.connList[(size_t)k * 4 + a];
      int ranks = 0;
      for (int b = 0; b < 4; b++) ranks |= (rec[a * 4 + b] & 0x7f) << (8 * b);
      const int j = fill[r]++;
      ent[2 * (size_t)j] = (k << 2) | a;
      ent[2 * (size_t)j + 1] = ranks;
    }
  }
  std::vector<int> chunk(1, 0);
  int rows = 0;
  int64_t blocks = 0;
  for (int r = 0; r < N; r++) {
    const int64_t len = hp.rowp[r + 1] - hp.rowp[r];
    if (rows == kRowChunkRows || blocks + len > kRowChunkBlocks) {
      chunk.push_back(r);
      rows = 0;
      blocks = 0;
    }
    rows++;
    blocks += len;
  }
  chunk.push_back(N);
  hp.rowElemPtr.swap(ptr);
  hp.rowElem.swap(ent);
  hp.rowChunk.swap(chunk);
}

// Pair layout (HostPlan::pairColourPtr ...).  Element f is e's right neighbour when
// f's nodes (0, ly) are e's nodes (P, ly) for every ly (tensor order: local node
// a = ly (P + 1) + lx); elements are paired greedily in id order.  Units (pairs
// and unpaired elements) are coloured greedily like the elements of the colour
// layout; codes are computed per colour with the units in parallel (they share no
// node) and the two elements of a pair in order.  Leaves the layout empty when
// the units need more than 64 colours.
static void build_pair_plan(const int *connPtr, const int *conn, HostPlan &hp) {
  const int P = hp.order, P1 = P + 1, nn = hp.nn, nE = hp.numElements;
  auto node = [&](int e, int lx, int ly) { return conn[connPtr[e] + ly * P1 + lx]; };
  auto key = [](int a, int b) { return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b; };
  // left edge (corner nodes (0, 0), (0, P)) -> element, sorted for lookup
  std::vector<std::pair<uint64_t, int>> left((size_t)nE);
  for (int e = 0; e < nE; e++) left[e] = {key(node(e, 0, 0), node(e, 0, P)), e};
  std::sort(left.begin(), left.end());
  std::vector<int> partner((size_t)nE, -1);
  std::vector<char> lead((size_t)nE, 0);
  for (int e = 0; e < nE; e++) {
    if (partner[e] >= 0) continue;
    const uint64_t k = key(node(e, P, 0), node(e, P, P));
    auto it = std::lower_bound(left.begin(), left.end(), std::make_pair(k, INT_MIN));
    if (it == left.end() || it->first != k) continue;
    if (it + 1 != left.end() && (it + 1)->first == k) continue;  // two elements share that left edge
    const int f = it->second;
    if (f == e || partner[f] >= 0) continue;
    bool same = true;
    for (int ly = 0; ly <= P && same; ly++) same = node(e, P, ly) == node(f, 0, ly);
    if (!same) continue;
    partner[e] = f;
    partner[f] = e;
    lead[e] = 1;
  }
  // units in order of their lead element, coloured greedily over node bit masks
  std::vector<int> unitLead, unitColour;
  std::vector<uint64_t> used((size_t)hp.numNodes, 0);
  int nc = 0;
  for (int e = 0; e < nE; e++) {
    if (partner[e] >= 0 && !lead[e]) continue;
    uint64_t m = 0;
    for (int w = 0; w < (partner[e] >= 0 ? 2 : 1); w++) {
      const int x = w ? partner[e] : e;
      for (int i = connPtr[x]; i < connPtr[x + 1]; i++) m |= used[conn[i]];
    }
    if (~m == 0) return;  // more than 64 colours: no pair layout
    const int c = __builtin_ctzll(~m);
    nc = std::max(nc, c + 1);
    for (int w = 0; w < (partner[e] >= 0 ? 2 : 1); w++) {
      const int x = w ? partner[e] : e;
      for (int i = connPtr[x]; i < connPtr[x + 1]; i++) used[conn[i]] |= (1ull << c);
    }
    unitLead.push_back(e);
    unitColour.push_back(c);
  }
  // per colour: pairs, then unpaired elements
  std::vector<int64_t> pairsOf((size_t)nc, 0), singlesOf((size_t)nc, 0);
  for (size_t u = 0; u < unitLead.size(); u++)
    (partner[unitLead[u]] >= 0 ? pairsOf : singlesOf)[unitColour[u]]++;
  hp.pairColourPtr.assign((size_t)nc + 1, 0);
  for (int c = 0; c < nc; c++) hp.pairColourPtr[c + 1] = hp.pairColourPtr[c] + (int)(2 * pairsOf[c] + singlesOf[c]);
  hp.pairList.assign((size_t)nE, -1);
  std::vector<int64_t> fillP((size_t)nc), fillS((size_t)nc);
  for (int c = 0; c < nc; c++) {
    fillP[c] = hp.pairColourPtr[c];
    fillS[c] = hp.pairColourPtr[c] + 2 * pairsOf[c];
  }
  // unit start positions (a pair's two elements are consecutive)
  std::vector<int64_t> unitPos(unitLead.size());
  for (size_t u = 0; u < unitLead.size(); u++) {
    const int e = unitLead[u], c = unitColour[u];
    if (partner[e] >= 0) {
      unitPos[u] = fillP[c];
      hp.pairList[fillP[c]++] = e;
      hp.pairList[fillP[c]++] = partner[e];
    } else {
      unitPos[u] = fillS[c];
      hp.pairList[fillS[c]++] = e;
    }
  }
  hp.pairConnList.resize((size_t)nE * nn);
  hp.pairCode.assign((size_t)nE * hp.codeStride, 0);
  std::vector<uint8_t> blockWritten((size_t)hp.nnzb, 0), nodeWritten((size_t)hp.numNodes, 0);
  // units grouped by colour, in list order
  std::vector<std::vector<int>> byColour((size_t)nc);
  for (size_t u = 0; u < unitLead.size(); u++) byColour[unitColour[u]].push_back((int)u);
  for (int c = 0; c < nc; c++) {
    const std::vector<int> &units = byColour[c];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)units.size(); i++) {
      const int u = units[i];
      const int e0 = unitLead[u];
      const int n = partner[e0] >= 0 ? 2 : 1;
      for (int w = 0; w < n; w++) {
        const int64_t k = unitPos[u] + w;
        const int e = hp.pairList[k];
        const int *en = conn + connPtr[e];
        int *cl = &hp.pairConnList[(size_t)k * nn];
        uint8_t *rec = &hp.pairCode[(size_t)k * hp.codeStride];
        for (int a = 0; a < nn; a++) cl[a] = en[a];
        for (int a = 0; a < nn; a++) {
          const int r = en[a];
          rec[nn * nn + a] = nodeWritten[r] ? 0 : 1;
          nodeWritten[r] = 1;
          const int *c0 = hp.cols.data() + hp.rowp[r], *c1 = hp.cols.data() + hp.rowp[r + 1];
          for (int b = 0; b < nn; b++) {
            const int *pos = std::lower_bound(c0, c1, en[b]);  // present: the colour layout found it
            uint8_t &bf = blockWritten[(size_t)(pos - hp.cols.data())];
            rec[a * nn + b] = (uint8_t)((pos - c0) | (bf ? 0 : 0x80));
            bf = 1;
          }
        }
      }
    }
  }
  hp.numPairColours = nc;
  hp.pairRegionEnd.resize((size_t)nc);
  for (int c = 0; c < nc; c++) hp.pairRegionEnd[c] = hp.pairColourPtr[c] + (int)(2 * pairsOf[c]);
  int64_t np = 0;
  for (int c = 0; c < nc; c++) np += pairsOf[c];
  hp.numPairs = np;
}

int build_host_plan(int order, int numNodes, const int *connPtr, const int *conn, int numElements, HostPlan &hp) {
  const int nn = (order + 1) * (order + 1);
  int st = validate_mesh(numNodes, connPtr, conn, numElements);
  if (st) return st;
  for (int e = 0; e < numElements; e++)
    if (connPtr[e + 1] - connPtr[e] != nn)
      return fail(FEM_ERR_INVALID_ARGUMENT, "element %d has %d nodes, order %d needs %d", e,
                  connPtr[e + 1] - connPtr[e], order, nn);
  hp.order = order;
  hp.nn = nn;
  hp.numNodes = numNodes;
  hp.numElements = numElements;
  hp.rowp.resize((size_t)numNodes + 1);
  st = build_pattern(numNodes, connPtr, conn, numElements, hp.rowp.data(), nullptr, &hp.nnzb);
  if (st) return st;
  hp.cols.resize((size_t)hp.nnzb);
  st = build_pattern(numNodes, connPtr, conn, numElements, hp.rowp.data(), hp.cols.data(), &hp.nnzb);
  if (st) return st;

  std::vector<int> colour((size_t)numElements);
  st = colour_greedy(numNodes, connPtr, conn, numElements, colour.data(), &hp.numColours);
  if (st) return st;
  hp.colourPtr.assign((size_t)hp.numColours + 1, 0);
  for (int e = 0; e < numElements; e++) hp.colourPtr[colour[e] + 1]++;
  for (int c = 0; c < hp.numColours; c++) hp.colourPtr[c + 1] += hp.colourPtr[c];
  hp.elemList.resize((size_t)numElements);
  {
    std::vector<int> fill(hp.colourPtr.begin(), hp.colourPtr.end() - 1);
    for (int e = 0; e < numElements; e++) hp.elemList[fill[colour[e]]++] = e;
  }
  hp.connList.resize((size_t)numElements * nn);
  hp.codeStride = (nn * nn + nn + 15) / 16 * 16;
  hp.blockCode.assign((size_t)numElements * hp.codeStride, 0);
  std::vector<uint8_t> blockWritten((size_t)hp.nnzb, 0), nodeWritten((size_t)numNodes, 0);
  int bad = 0;
  for (int c = 0; c < hp.numColours; c++) {
    // Elements of one colour share no node, hence no block: the byte flags they
    // touch are disjoint and the loop is race-free.
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int k = hp.colourPtr[c]; k < hp.colourPtr[c + 1]; k++) {
      const int e = hp.elemList[k];
      const int *en = conn + connPtr[e];
      int *cl = &hp.connList[(size_t)k * nn];
      for (int a = 0; a < nn; a++) cl[a] = en[a];
      for (int a = 0; a < nn; a++) {
        const int r = en[a];
        uint8_t &nf = nodeWritten[r];
        uint8_t *rec = &hp.blockCode[(size_t)k * hp.codeStride];
        rec[nn * nn + a] = nf ? 0 : 1;
        nf = 1;
        const int *c0 = hp.cols.data() + hp.rowp[r], *c1 = hp.cols.data() + hp.rowp[r + 1];
        for (int b = 0; b < nn; b++) {
          const int *pos = std::lower_bound(c0, c1, en[b]);
          const int64_t rank = pos - c0;
          if (pos == c1 || *pos != en[b] || rank > 127) {
            bad = 1;
            continue;
          }
          uint8_t &bf = blockWritten[(size_t)(pos - hp.cols.data())];
          rec[a * nn + b] = (uint8_t)(rank | (bf ? 0 : 0x80));
          bf = 1;
        }
      }
    }
  }
  if (bad) return fail(FEM_ERR_UNSUPPORTED, "a BSR row holds more than 128 blocks; use the map-based entry points");
  if (order == 1) build_row_plan(hp);
  if (order >= 2) build_pair_plan(connPtr, conn, hp);
  return FEM_SUCCESS;
}

}  // namespace fem

extern "C" {

const char *fem_last_error(void) { return fem::last_error_cstr(); }

const char *fem_status_string(int status) {
  switch (status) {
    case FEM_SUCCESS: return "success";
    case FEM_ERR_INVALID_ORDER: return "element order must be 1..4";
    case FEM_ERR_INVALID_ARGUMENT: return "invalid argument";
    case FEM_ERR_MISALIGNED: return "array not 16-byte aligned";
    case FEM_ERR_CUDA: return "CUDA runtime error";
    case FEM_ERR_OVERFLOW: return "index overflows int32";
    case FEM_ERR_NOT_FOUND: return "element block missing from BSR pattern";
    case FEM_ERR_UNSUPPORTED: return "unsupported input";
    case FEM_ERR_BUDGET: return "device memory budget exhausted";
    case FEM_ERR_TIMEOUT: return "a bounded in-kernel wait ran out";
    default: return "unknown status";
  }
}

int fem_version(void) { return 100; }

int fem_build_bsr_pattern(int numNodes, const int *connPtr, const int *conn, int numElements, int *rowp, int *cols,
                          int64_t *nnzb) {
  fem::clear_error();
  return fem::build_pattern(numNodes, connPtr, conn, numElements, rowp, cols, nnzb);
}

int fem_build_element_bsr_map(const int *connPtr, const int *conn, int numElements, int nodesPerElement,
                              const int *rowp, const int *cols, int *map) {
  fem::clear_error();
  if (numElements < 0 || nodesPerElement <= 0) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "bad sizes");
  if (numElements == 0) return FEM_SUCCESS;
  if (!connPtr || !conn || !rowp || !cols || !map) return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL array");
  const int n = nodesPerElement;
  int status = FEM_SUCCESS;
#pragma omp parallel for schedule(static) reduction(max : status)
  for (int e = 0; e < numElements; e++) {
    const int *en = conn + connPtr[e];
    for (int a = 0; a < n; a++) {
      const int *c0 = cols + rowp[en[a]], *c1 = cols + rowp[en[a] + 1];
      for (int b = 0; b < n; b++) {
        const int *pos = std::lower_bound(c0, c1, en[b]);
        if (pos == c1 || *pos != en[b]) {
          status = std::max(status, (int)FEM_ERR_NOT_FOUND);
          continue;
        }
        const int64_t off = (int64_t)(pos - cols) * 4;
        if (off > INT_MAX) {
          status = std::max(status, (int)FEM_ERR_OVERFLOW);
          continue;
        }
        map[((int64_t)e * n + a) * n + b] = (int)off;
      }
    }
  }
  if (status == FEM_ERR_NOT_FOUND) return fem::fail(status, "an element block is not in the BSR pattern");
  if (status == FEM_ERR_OVERFLOW) return fem::fail(status, "block offset*4 exceeds INT32_MAX");
  return status;
}

int fem_colour_elements(int numNodes, const int *connPtr, const int *conn, int numElements, int *colour,
                        int *numColours) {
  fem::clear_error();
  return fem::colour_greedy(numNodes, connPtr, conn, numElements, colour, numColours);
}

int fem_pair_layout(int elementOrder, int numNodes, const int *connPtr, const int *conn, int numElements,
                    int *elemList, int *colourPtr, int *numColours, int64_t *numPairs, uint8_t *codes,
                    int *codeStride) {
  fem::clear_error();
  if (!elemList || !colourPtr || !numColours || !numPairs)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL output");
  if (elementOrder < 2 || elementOrder > 4)
    return fem::fail(FEM_ERR_INVALID_ORDER, "pair layout: orders 2..4 (order %d)", elementOrder);
  fem::HostPlan hp;
  int st = fem::build_host_plan(elementOrder, numNodes, connPtr, conn, numElements, hp);
  if (st) return st;
  *numColours = hp.numPairColours;
  *numPairs = hp.numPairs;
  if (codeStride) *codeStride = hp.codeStride;
  if (hp.numPairColours == 0) return FEM_SUCCESS;
  std::copy(hp.pairList.begin(), hp.pairList.end(), elemList);
  std::copy(hp.pairColourPtr.begin(), hp.pairColourPtr.end(), colourPtr);
  if (codes) std::copy(hp.pairCode.begin(), hp.pairCode.end(), codes);
  return FEM_SUCCESS;
}

}  // extern "C"
