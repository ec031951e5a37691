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
  // Orders 2-4, pair layout of the fragment kernel's single-mesh assembly: elements
  // paired with the neighbour across their right edge (its left edge, node for
  // node), pairs coloured so that the pairs of one colour share no node, each
  // colour listing its pairs (two consecutive positions, the pair's first element
  // first) and then its unpaired elements.  Codes as above, in list order, so the
  // second element of a pair adds to the blocks and residual rows of the shared
  // edge that the first one stored.
  int numPairColours = 0;
  int64_t numPairs = 0;
  std::vector<int> pairColourPtr, pairList, pairConnList;
  std::vector<int> pairRegionEnd;  // per colour: the end of its pairs (its unpaired elements follow)
  std::vector<uint8_t> pairCode;
};
constexpr int kRowChunkRows = 32, kRowChunkBlocks = 320;
int build_host_plan(int order, int numNodes, const int *connPtr, const int *conn, int numElements, HostPlan &hp);

}  // namespace fem
