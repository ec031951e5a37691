// Patch layout of an order-3 assembly plan (host side, integer work only).
//
// The colour-ordered plan writes every element's 2x2 blocks on their own: runs of
// four 32-byte blocks at arbitrary offsets, neighbouring runs of a matrix row written
// by other elements in other launches.  A patch groups neighbouring elements (on a
// structured mesh, consecutive element ids form a strip along a grid row) so that one
// CTA sums their blocks in shared memory and writes each matrix row once, as a few
// long contiguous segments.  This file builds, from the plan's pattern and block
// ranks:
//   * the patches, greedily in element order: an element joins the open patch in the
//     first phase (0, then 1) none of whose elements shares a node with it, while the
//     phase has room (four elements) and the patch's slot and node budgets hold;
//   * the patch colouring (greedy, patches sharing a node get different colours);
//   * per patch: the slot layout (rows in ascending node order, each row a slot range
//     covering the ranks it receives), the code records and slot bases of its element
//     positions, the store/add segments of its blocks (maximal runs contiguous both
//     in the BSR values and in the slots, with one mode) and its residual rows.
// The same steps restated in Python check the tables (tests/test_patch_layout.py).
#include <algorithm>
#include <climits>
#include <vector>

#include "fem_common.h"

namespace fem {

namespace {

// Patch formation over the elements in id order; fills `elem` (kPatchElems per patch).
int form_patches(const HostPlan &hp, const int *connPtr, const int *conn, const std::vector<int> &pos,
                 std::vector<int> &elem) {
  const int nn = hp.nn, cs = hp.codeStride;
  std::vector<uint8_t> mark((size_t)hp.numNodes, 0);  // bit p: node of a phase-p element; 4: in the patch
  std::vector<int> lo((size_t)hp.numNodes, 0), hi((size_t)hp.numNodes, 0);
  std::vector<int> open;
  int cur[kPatchElems], cnt[2] = {0, 0}, slots = 0;
  std::fill(cur, cur + kPatchElems, -1);
  auto close = [&] {
    elem.insert(elem.end(), cur, cur + kPatchElems);
    for (int r : open) mark[r] = 0;
    open.clear();
    std::fill(cur, cur + kPatchElems, -1);
    cnt[0] = cnt[1] = slots = 0;
  };
  std::vector<int> rmin(nn), rmax(nn);
  for (int e = 0; e < hp.numElements; e++) {
    const int *en = conn + connPtr[e];
    const uint8_t *rec = &hp.blockCode[(size_t)pos[e] * cs];
    for (int a = 0; a < nn; a++) {
      int mn = INT_MAX, mx = -1;
      for (int b = 0; b < nn; b++) {
        const int k = rec[a * nn + b] & 0x7f;
        mn = std::min(mn, k);
        mx = std::max(mx, k);
      }
      rmin[a] = mn;
      rmax[a] = mx;
    }
    for (int attempt = 0; attempt < 2; attempt++) {
      bool ok[2] = {cnt[0] < kPatchElems / 2, cnt[1] < kPatchElems / 2};
      for (int a = 0; a < nn; a++) {
        if (mark[en[a]] & 1) ok[0] = false;
        if (mark[en[a]] & 2) ok[1] = false;
      }
      const int ph = ok[0] ? 0 : (ok[1] ? 1 : -1);
      if (ph >= 0) {
        int ns = slots, nodes = (int)open.size();
        for (int a = 0; a < nn; a++) {
          const int r = en[a];
          if (mark[r]) {
            ns += std::max(hi[r], rmax[a]) - std::min(lo[r], rmin[a]) - (hi[r] - lo[r]);
          } else {
            ns += rmax[a] - rmin[a] + 1;
            nodes++;
          }
        }
        if (ns <= kPatchSlots && nodes <= kPatchNodes) {
          cur[2 * cnt[ph] + ph] = e;
          cnt[ph]++;
          slots = ns;
          for (int a = 0; a < nn; a++) {
            const int r = en[a];
            if (!mark[r]) {
              open.push_back(r);
              lo[r] = rmin[a];
              hi[r] = rmax[a];
            } else {
              lo[r] = std::min(lo[r], rmin[a]);
              hi[r] = std::max(hi[r], rmax[a]);
            }
            mark[r] |= (uint8_t)(4 | (1 << ph));
          }
          break;
        }
      }
      if (attempt == 1 || cnt[0] + cnt[1] == 0)
        return fail(FEM_ERR_UNSUPPORTED, "element %d does not fit one patch (%d slots, %d nodes)", e, kPatchSlots,
                    kPatchNodes);
      close();
    }
  }
  if (cnt[0] + cnt[1] > 0) close();
  return FEM_SUCCESS;
}

// Segment and residual-row lists of one patch, concatenated after the colour loop.
struct PatchTables {
  std::vector<int> seg, node;
};

}  // namespace

int build_patch_plan(const HostPlan &hp, const int *connPtr, const int *conn, PatchPlan &pp) {
  const int nn = hp.nn, cs = hp.codeStride, PE = kPatchElems;
  if (hp.order != 3) return fail(FEM_ERR_UNSUPPORTED, "patch assembly is built for order 3 (order %d)", hp.order);
  if (hp.nnzb >= INT_MAX) return fail(FEM_ERR_OVERFLOW, "patch segments index blocks as int32 (nnzb %lld)",
                                      (long long)hp.nnzb);
  std::vector<int> pos((size_t)hp.numElements);
  for (int k = 0; k < hp.numElements; k++) pos[hp.elemList[k]] = k;
  std::vector<int> formed;
  int st = form_patches(hp, connPtr, conn, pos, formed);
  if (st) return st;
  const int np = (int)(formed.size() / PE);

  // nodes of each patch (sorted, unique) and node -> patches
  std::vector<int64_t> pnPtr((size_t)np + 1, 0);
  std::vector<int> pn;
  {
    std::vector<int> buf;
    for (int p = 0; p < np; p++) {
      buf.clear();
      for (int j = 0; j < PE; j++) {
        const int e = formed[(size_t)p * PE + j];
        if (e >= 0) buf.insert(buf.end(), conn + connPtr[e], conn + connPtr[e] + nn);
      }
      std::sort(buf.begin(), buf.end());
      buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
      pn.insert(pn.end(), buf.begin(), buf.end());
      pnPtr[p + 1] = (int64_t)pn.size();
    }
  }
  // greedy colouring in formation order: a patch takes the lowest colour no earlier
  // patch sharing one of its nodes holds
  std::vector<int> colour((size_t)np);
  {
    std::vector<uint64_t> used((size_t)hp.numNodes, 0);
    int nc = 0;
    for (int p = 0; p < np; p++) {
      uint64_t m = 0;
      for (int64_t i = pnPtr[p]; i < pnPtr[p + 1]; i++) m |= used[pn[(size_t)i]];
      if (~m == 0) return fail(FEM_ERR_UNSUPPORTED, "patch %d needs more than 64 colours", p);
      const int c = __builtin_ctzll(~m);
      colour[p] = c;
      nc = std::max(nc, c + 1);
      for (int64_t i = pnPtr[p]; i < pnPtr[p + 1]; i++) used[pn[(size_t)i]] |= 1ull << c;
    }
    pp.numColours = nc;
  }
  pp.numPatches = np;
  pp.colourPtr.assign((size_t)pp.numColours + 1, 0);
  for (int p = 0; p < np; p++) pp.colourPtr[colour[p] + 1]++;
  for (int c = 0; c < pp.numColours; c++) pp.colourPtr[c + 1] += pp.colourPtr[c];
  std::vector<int> order((size_t)np);  // patch order: by colour, formation order within
  {
    std::vector<int> fill(pp.colourPtr.begin(), pp.colourPtr.end() - 1);
    for (int p = 0; p < np; p++) order[fill[colour[p]]++] = p;
  }

  pp.elem.resize((size_t)np * PE);
  pp.connList.assign((size_t)np * PE * nn, -1);
  pp.code.assign((size_t)np * PE * cs, 0);
  pp.rb.assign((size_t)np * PE * nn, 0);
  std::vector<PatchTables> tabs((size_t)np);
  std::vector<uint8_t> blockWritten((size_t)hp.nnzb, 0), nodeWritten((size_t)hp.numNodes, 0);
  int bad = 0;
  for (int c = 0; c < pp.numColours; c++) {
    // patches of one colour share no node, hence no block: the flags they touch are disjoint
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
    for (int q = pp.colourPtr[c]; q < pp.colourPtr[c + 1]; q++) {
      const int p = order[q];
      const int *nodes = pn.data() + pnPtr[p];
      const int nnodes = (int)(pnPtr[p + 1] - pnPtr[p]);
      auto local = [&](int r) { return (int)(std::lower_bound(nodes, nodes + nnodes, r) - nodes); };
      const int *el = formed.data() + (size_t)p * PE;
      // rank range of every patch row, slot bases (rows in ascending node order)
      std::vector<int> lo(nnodes, INT_MAX), hi(nnodes, -1), owner(nnodes, -1), base(nnodes);
      for (int j = 0; j < PE; j++) {
        if (el[j] < 0) continue;
        const int *en = conn + connPtr[el[j]];
        const uint8_t *rec = &hp.blockCode[(size_t)pos[el[j]] * cs];
        for (int a = 0; a < nn; a++) {
          const int l = local(en[a]);
          if (j % 2 == 0) owner[l] = j;
          for (int b = 0; b < nn; b++) {
            const int k = rec[a * nn + b] & 0x7f;
            lo[l] = std::min(lo[l], k);
            hi[l] = std::max(hi[l], k);
          }
        }
      }
      int slots = 0;
      for (int l = 0; l < nnodes; l++) {
        base[l] = slots - lo[l];
        slots += hi[l] - lo[l] + 1;
      }
      if (slots > kPatchSlots || nnodes > kPatchNodes) bad = 1;
      // element positions: node ids, code records, slot bases
      std::vector<std::pair<int64_t, int>> blocks;  // (block index, slot)
      for (int j = 0; j < PE; j++) {
        const size_t P = (size_t)q * PE + j;
        pp.elem[P] = el[j];
        if (el[j] < 0) continue;
        const int *en = conn + connPtr[el[j]];
        const uint8_t *rec = &hp.blockCode[(size_t)pos[el[j]] * cs];
        uint8_t *out = &pp.code[P * cs];
        int lid[32];
        for (int a = 0; a < nn; a++) lid[a] = local(en[a]);
        for (int a = 0; a < nn; a++) {
          const int l = lid[a];
          pp.connList[P * nn + a] = en[a];
          pp.rb[P * nn + a] = base[l] * 256 + l;
          // phase 1: added where the phase-0 element holding node a (if any) holds node b too
          const int own = (j % 2 == 1) ? owner[l] : -1;
          out[nn * nn + a] = own >= 0 ? 1 : 0;
          for (int b = 0; b < nn; b++) {
            const int k = rec[a * nn + b] & 0x7f;
            const bool add = own >= 0 && owner[lid[b]] == own;
            out[a * nn + b] = (uint8_t)(k | (add ? 0x80 : 0));
            blocks.emplace_back((int64_t)hp.rowp[en[a]] + k, base[l] + k);
          }
        }
      }
      std::sort(blocks.begin(), blocks.end());
      blocks.erase(std::unique(blocks.begin(), blocks.end()), blocks.end());
      // segments: runs contiguous in the values and in the slots, one mode each
      PatchTables &T = tabs[(size_t)q];
      int64_t g0 = -2;
      int s0 = 0, n = 0, m0 = 0;
      auto flush = [&] {
        if (n > 0) {
          T.seg.push_back((int)g0);
          T.seg.push_back((int)((unsigned)s0 | ((unsigned)n << 16) | ((unsigned)m0 << 31)));
        }
      };
      for (const auto &bs : blocks) {
        const int m = blockWritten[(size_t)bs.first] ? 1 : 0;
        if (n > 0 && bs.first == g0 + n && bs.second == s0 + n && m == m0 && n < kPatchSegMax) {
          n++;
        } else {
          flush();
          g0 = bs.first;
          s0 = bs.second;
          m0 = m;
          n = 1;
        }
      }
      flush();
      for (const auto &bs : blocks) blockWritten[(size_t)bs.first] = 1;
      for (int l = 0; l < nnodes; l++) {
        const int r = nodes[l];
        T.node.push_back(r | (nodeWritten[r] ? INT_MIN : 0));
        nodeWritten[r] = 1;
      }
    }
  }
  if (bad) return fail(FEM_ERR_UNSUPPORTED, "patch layout exceeds its shared-memory budget");
  pp.segPtr.assign((size_t)np + 1, 0);
  pp.nodePtr.assign((size_t)np + 1, 0);
  for (int q = 0; q < np; q++) {
    pp.segPtr[q + 1] = pp.segPtr[q] + (int)tabs[q].seg.size() / 2;
    pp.nodePtr[q + 1] = pp.nodePtr[q] + (int)tabs[q].node.size();
  }
  pp.seg.resize((size_t)pp.segPtr[np] * 2);
  pp.node.resize((size_t)pp.nodePtr[np]);
  for (int q = 0; q < np; q++) {
    std::copy(tabs[q].seg.begin(), tabs[q].seg.end(), pp.seg.begin() + 2 * (size_t)pp.segPtr[q]);
    std::copy(tabs[q].node.begin(), tabs[q].node.end(), pp.node.begin() + pp.nodePtr[q]);
  }
  return FEM_SUCCESS;
}

}  // namespace fem

extern "C" int fem_patch_layout(int elementOrder, int numNodes, const int *connPtr, const int *conn, int numElements,
                                int *numPatches, int *numColours, int64_t *numSegments, int64_t *numPatchNodes,
                                int *colourPtr, int *patchElem, uint8_t *code, int *slotBase, int *segPtr, int *seg,
                                int *nodePtr, int *node) {
  fem::clear_error();
  if (elementOrder != 3) return fem::fail(FEM_ERR_UNSUPPORTED, "patch layout: order 3 only (order %d)", elementOrder);
  if (!numPatches || !numColours || !numSegments || !numPatchNodes)
    return fem::fail(FEM_ERR_INVALID_ARGUMENT, "NULL size argument");
  fem::HostPlan hp;
  int st = fem::build_host_plan(elementOrder, numNodes, connPtr, conn, numElements, hp);
  if (st) return st;
  fem::PatchPlan pp;
  if ((st = fem::build_patch_plan(hp, connPtr, conn, pp))) return st;
  *numPatches = pp.numPatches;
  *numColours = pp.numColours;
  *numSegments = (int64_t)pp.seg.size() / 2;
  *numPatchNodes = (int64_t)pp.node.size();
  auto put = [](auto *dst, const auto &v) {
    if (dst) std::copy(v.begin(), v.end(), dst);
  };
  put(colourPtr, pp.colourPtr);
  put(patchElem, pp.elem);
  put(code, pp.code);
  put(slotBase, pp.rb);
  put(segPtr, pp.segPtr);
  put(seg, pp.seg);
  put(nodePtr, pp.nodePtr);
  put(node, pp.node);
  return FEM_SUCCESS;
}
