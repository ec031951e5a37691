// Shared internals of libfemb200: error reporting and small helpers.
#pragma once

#include <cstdint>
#include <cstdio>
#include <vector>

#include "fem_b200.h"

namespace fem {

// Records a message for fem_last_error() on this host thread and returns `status`.
int fail(int status, const char *fmt, ...);
void clear_error();
const char *last_error_cstr();

inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Host builders (fem_host.cpp).
int build_pattern(int numNodes, const int *connPtr, const int *conn, int numElements, int *rowp, int *cols,
                  int64_t *nnzb);
int colour_greedy(int numNodes, const int *connPtr, const int *conn, int numElements, int *colour,
                  int *numColours);

// Plan topology built on the host before upload (fem_host.cpp).
struct HostPlan {
  int order = 0, nn = 0, numNodes = 0, numElements = 0, numColours = 0;
  int64_t nnzb = 0;
  std::vector<int> rowp, cols;                // pattern
  std::vector<int> elemList;            // elements in colour order
  std::vector<int> colourPtr;           // numColours+1 offsets into elemList
  std::vector<int> connList;            // conn in elemList order, nn per element
  // Per listed element k a record of codeStride bytes: [a*nn + b] = rank of the
  // block (a, b) in row conn[a] | 0x80 when this element stores it first, then
  // [nn*nn + a] = 1 when this element writes node a's residual first; zero padding
  // to a multiple of 16 bytes (records are copied to shared memory in 16-byte chunks).
  int codeStride = 0;
  std::vector<uint8_t> blockCode;
  // Order 1, row assembly (each block row written once by the warp that owns it):
  // rowElemPtr[numNodes+1] indexes rowElem, two ints per (node r, element k listing
  // r): {k << 2 | a (local index of r), ranks of the element's four nodes in row r,
  // one byte each}; rowChunk[numChunks+1] cuts the rows into chunks of at most
  // kRowChunkRows rows and kRowChunkBlocks blocks.  Empty when not applicable.
  std::vector<int> rowElemPtr, rowElem, rowChunk;
};
constexpr int kRowChunkRows = 32, kRowChunkBlocks = 320;
int build_host_plan(int order, int numNodes, const int *connPtr, const int *conn, int numElements, HostPlan &hp);

// Patch layout (order 3, fem_patch.cpp).  A patch is up to kPatchElems elements
// that one CTA assembles into a shared-memory copy of the matrix blocks and
// residual rows they touch, then writes out as contiguous row segments.  Position
// j of a patch belongs to warp j/2 and phase j%2: the elements of one phase share
// no node, so a block or residual row receives at most one contribution per phase
// (phase 0 stores it, phase 1 stores or adds).  Patches of one colour share no
// node; colours run in order, the first colour touching a block stores it and
// later ones add.
constexpr int kPatchElems = 8, kPatchSlots = 2560, kPatchNodes = 128, kPatchSegMax = 1024;
struct PatchPlan {
  int numPatches = 0, numColours = 0;
  std::vector<int> colourPtr;  // numColours+1 offsets into the patch order
  std::vector<int> elem;       // [patch][kPatchElems] element id, -1 for an empty position
  std::vector<int> connList;   // [patch][position][nn] node ids (-1 for an empty position)
  // [patch][position] code record of HostPlan::codeStride bytes: [a*nn + b] = rank of
  // block (a, b) in row conn[a] | 0x80 when it is added to the patch copy (phase 1,
  // a phase-0 element holds the same block); [nn*nn + a] = 1 when node a's residual
  // is added.
  std::vector<uint8_t> code;
  // [patch][position][nn]: slot base * 256 + patch-local index of node a; the block
  // (a, b) sits in slot base + rank, the residual of node a in residual slot index.
  std::vector<int> rb;
  std::vector<int> segPtr;  // numPatches+1 offsets into seg
  // two ints per segment: first block index in the BSR values, slot | count << 16 |
  // 1 << 31 when the segment is added (an earlier colour stored it)
  std::vector<int> seg;
  std::vector<int> nodePtr;  // numPatches+1 offsets into node (patch-local nodes, ascending)
  std::vector<int> node;     // node id | 1 << 31 when the residual row is added
};
int build_patch_plan(const HostPlan &hp, const int *connPtr, const int *conn, PatchPlan &pp);

}  // namespace fem
