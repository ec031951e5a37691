/*
 * fem_b200.h -- C ABI of the B200 plane-stress quad assembly library (libfemb200.so).
 *
 * Global residual and 2x2-block BSR Jacobian assembly for 2D plane-stress
 * Lagrange quadrilaterals of order 1..4, (p+1)x(p+1) Gauss points, linear
 * strain.  All array arguments are plain pointers; no C++ or torch types cross
 * this boundary.
 *
 * Conventions shared with A-CGray/GPU-FEM-Project (element/FEKernels.h):
 *   - nodeCoords[node*2 + d] and states[node*2 + s]: node-major, 2 values per node.
 *   - connPtr (CSR offsets) and conn (int32 node ids); element e's local node
 *     a = ay*(p+1) + ax is conn[connPtr[e] + a] (tensor-product order).
 *   - residual[node*2 + s]; BSR values are 2x2 row-major blocks:
 *     matEntries[blk*4 + i*2 + j] couples DOF (row node, i) with (col node, j).
 *   - elementBCSRMap[e*n*n + a*n + b] is the offset (in doubles, = block index*4)
 *     of the block coupling local nodes a and b (verification/TACSHelpers.h:133-137).
 *
 * Every entry point returns a status (FEM_SUCCESS == 0) instead of exiting the
 * process.  Device-side entry points take DEVICE pointers (as the reference's
 * nvcc build does), must be 16-byte aligned for coordinate/state/output arrays,
 * and are asynchronous on `stream` (a cudaStream_t, NULL = legacy default
 * stream) unless elapsedSeconds is non-NULL, in which case the call records
 * CUDA events around the launch, synchronises the stream and returns the
 * device time in seconds (the reference always synchronised and returned seconds).
 */
#ifndef FEM_B200_H
#define FEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------- */
#define FEM_SUCCESS 0
#define FEM_ERR_INVALID_ORDER 1    /* element order outside 1..4 (reference: silent no-op)   */
#define FEM_ERR_INVALID_ARGUMENT 2 /* NULL where data is required, negative sizes, ...      */
#define FEM_ERR_MISALIGNED 3       /* a double array is not 16-byte aligned                 */
#define FEM_ERR_CUDA 4             /* a CUDA runtime call failed; see fem_last_error()      */
#define FEM_ERR_OVERFLOW 5         /* an index does not fit the int32 format                */
#define FEM_ERR_NOT_FOUND 6        /* an element block is missing from the BSR pattern      */
#define FEM_ERR_UNSUPPORTED 7      /* input outside what this entry point supports          */
#define FEM_ERR_BUDGET 8           /* device-memory budget exhausted (serving admission)    */
#define FEM_ERR_TIMEOUT 9          /* a bounded in-kernel wait ran out (results invalid)     */

#define FEM_PRECISION_FP64 0  /* all element arithmetic in FP64                               */
#define FEM_PRECISION_MIXED 1 /* FP64 J/detJ/J^-1, weak stress and accumulate; element
                               stiffness in reduced precision: order 3 as BF16 tensor-core
                               products of three-way split operands (FP32 accumulate;
                               as fast as FP64 in the colour layout, ~12 % slower than
                               FP64 in a plan's pair layout, whose gain it does not
                               share), order 4 and the order-1 drop-in as FP32 element
                               products; orders 1-2 (plans) run the faster FP64 kernel
                               and the result is FP64 */

/* Strain measure of the weak residual: the reference's A2D::GreenStrainType
 * template option of planeStressWeakRes and the four assembly kernels
 * (element/FEKernels.h:286,317,379,589,786).  Its dispatchers always take the
 * default, LINEAR. */
#define FEM_STRAIN_LINEAR 0    /* eps = sym(du/dx); weakRes = w detJ t sigma                 */
#define FEM_STRAIN_NONLINEAR 1 /* Green strain E = 1/2 (g + g^T + g^T g), g = du/dx;        */
                               /* weakRes = w detJ t (I + g) S, S = 2 mu E + lambda tr(E) I  */

const char *fem_status_string(int status);
/* Message describing the last failure on the calling host thread ("" if none). */
const char *fem_last_error(void);
/* Library version: major*10000 + minor*100 + patch. */
int fem_version(void);

/* ---- drop-in entry points (device pointers, accumulate-into) -------------------------- */

/* Replaces runResidualKernel (element/FEKernels.h:1030-1102).  Adds the element
 * residuals into `residual` (the caller zeroes it first, as the reference's
 * driver does, verification/TestKernels.cpp:237). */
int fem_run_residual(int elementOrder, const int *connPtr, const int *conn, int numElements, const double *states,
                     const double *nodeCoords, double E, double nu, double t, double *residual, void *stream,
                     double *elapsedSeconds);

/* Replaces runJacobianKernel (element/FEKernels.h:1125-1225).  Adds the element
 * matrices into matEntries through elementBCSRMap and, when residual != NULL,
 * the element residuals into residual (FEKernels.h:996). */
int fem_run_jacobian(int elementOrder, const int *connPtr, const int *conn, int numElements, const double *states,
                     const double *nodeCoords, double E, double nu, double t, const int *elementBCSRMap,
                     double *residual, double *matEntries, void *stream, double *elapsedSeconds);

/* Same contracts as the two above with FEM_PRECISION_MIXED element arithmetic
 * (no reference counterpart: the reference is FP64 only). */
int fem_run_residual_mixed(int elementOrder, const int *connPtr, const int *conn, int numElements,
                           const double *states, const double *nodeCoords, double E, double nu, double t,
                           double *residual, void *stream, double *elapsedSeconds);
int fem_run_jacobian_mixed(int elementOrder, const int *connPtr, const int *conn, int numElements,
                           const double *states, const double *nodeCoords, double E, double nu, double t,
                           const int *elementBCSRMap, double *residual, double *matEntries, void *stream,
                           double *elapsedSeconds);

/* The reference kernels with an explicit strainType template argument
 * (assemblePlaneStressResidualKernel<order,2,2,strainType>, FEKernels.h:585-728;
 * assemblePlaneStressJacobianKernel<...,strainType>, FEKernels.h:782-1006), which
 * runResidualKernel/runJacobianKernel never expose.  Same contracts as
 * fem_run_residual / fem_run_jacobian.  precision: FEM_PRECISION_*; strainType:
 * FEM_STRAIN_*; FEM_STRAIN_NONLINEAR requires FEM_PRECISION_FP64
 * (FEM_ERR_INVALID_ARGUMENT otherwise). */
int fem_run_residual_ex(int elementOrder, const int *connPtr, const int *conn, int numElements, const double *states,
                        const double *nodeCoords, double E, double nu, double t, double *residual, int precision,
                        int strainType, void *stream, double *elapsedSeconds);
int fem_run_jacobian_ex(int elementOrder, const int *connPtr, const int *conn, int numElements, const double *states,
                        const double *nodeCoords, double E, double nu, double t, const int *elementBCSRMap,
                        double *residual, double *matEntries, int precision, int strainType, void *stream,
                        double *elapsedSeconds);

/* ---- host-side setup helpers (HOST pointers) ------------------------------------------- */

/* BSR sparsity of the nodal adjacency: row r lists, ascending, every node that
 * shares an element with node r (itself included).  This is the pattern TACS
 * hands the reference driver (verification/TestKernels.cpp:105-115).  Call with
 * cols == NULL to obtain *nnzb only; rowp has numNodes+1 entries. */
int fem_build_bsr_pattern(int numNodes, const int *connPtr, const int *conn, int numElements, int *rowp, int *cols,
                          int64_t *nnzb);

/* Replaces generateElementBCSRMap (verification/TACSHelpers.h:138-182):
 * map[e*n*n + a*n + b] = (position of conn[b] in row conn[a]) * 4.
 * FEM_ERR_NOT_FOUND if a block is missing, FEM_ERR_OVERFLOW if an offset
 * exceeds INT32_MAX. */
int fem_build_element_bsr_map(const int *connPtr, const int *conn, int numElements, int nodesPerElement,
                              const int *rowp, const int *cols, int *map);

/* Deterministic greedy element colouring in element order: no two elements of
 * one colour share a node.  colour has numElements entries.  (No reference
 * counterpart: the reference scatters with atomics only.) */
int fem_colour_elements(int numNodes, const int *connPtr, const int *conn, int numElements, int *colour,
                        int *numColours);
/* The pair layout a plan of order 2-4 builds for its single-mesh fragment-kernel
 * launches (fem_plan_set_layout), computed on the host: elemList[numElements]
 * (pairs first within each colour, a pair's elements consecutive),
 * colourPtr[numColours + 1] (at most 65 entries), the pairs formed and, when
 * codes != NULL, the code records (numElements * codeStride bytes: per listed
 * element, [a*nn + b] = rank of block (a, b) in row conn[a] | 0x80 for its first
 * contributor, [nn*nn + a] = 1 for the first writer of node a's residual).
 * numColours = 0: no pair layout (more than 64 colours).  (No reference counterpart.) */
int fem_pair_layout(int elementOrder, int numNodes, const int *connPtr, const int *conn, int numElements,
                    int *elemList, int *colourPtr, int *numColours, int64_t *numPairs, uint8_t *codes,
                    int *codeStride);

/* y = A x for a 2x2-block BSR matrix on the device (rowp/cols/A/x/y device
 * pointers).  Consumer of the assembled Jacobian (the reference exports the
 * same BCSR layout to TACS, verification/TestKernels.cpp:113-121). */
int fem_bsr_spmv(int numRows, const int *rowp, const int *cols, const double *A, const double *x, double *y,
                 void *stream);

/* ---- assembly plans: overwrite semantics, colour-ordered, no map ---------------------- */
/* A plan owns device copies of the mesh topology, its BSR pattern, an element
 * colouring and compact per-element block codes.  fem_plan_assemble writes the
 * COMPLETE residual and matrix (the caller zeroes nothing): colours run in
 * order, no two elements of one colour share a node, the first contributor to
 * each block stores it and later colours add to it.  (No reference counterpart.) */
typedef struct fem_plan fem_plan;

int fem_plan_create(int elementOrder, int numNodes, const int *connPtr, const int *conn, int numElements,
                    fem_plan **plan);
int fem_plan_destroy(fem_plan *plan);
/* Sizes: numNodes, numElements, nnzb, numColours, device bytes held. */
int fem_plan_info(const fem_plan *plan, int *numNodes, int *numElements, int64_t *nnzb, int *numColours,
                  int64_t *deviceBytes);
/* Copy the plan's BSR pattern to host arrays (rowp: numNodes+1, cols: nnzb). */
int fem_plan_get_pattern(const fem_plan *plan, int *rowp, int *cols);
/* Row chunks of an order-1 plan: > 0 when its LINEAR assembly runs as row
 * assembly (one launch, each block row written once), 0 when it runs by colours. */
int fem_plan_row_chunks(const fem_plan *plan, int *numChunks);
/* Element order of the single-mesh colour launches that the warp-fragment kernel
 * runs (orders 2-4; fem_plan_assemble without a schedule):
 *   FEM_LAYOUT_PAIRS    (default where built) each element is paired with the
 *                       neighbour across its right edge (that element's left edge,
 *                       node for node); pairs are coloured so that one colour's
 *                       pairs share no node, and a warp assembles a pair in one
 *                       step, the second element adding to the shared edge's
 *                       blocks the first one stored, so that the rows the two
 *                       share are written while their lines are in L2;
 *   FEM_LAYOUT_COLOURS  the element colouring above (what every other path runs).
 * The results agree to rounding: a block's contributions are added in another
 * order where more than two elements share it.  fem_plan_get_layout also reports
 * the pairs formed and their colours (0, 0 when the plan has no pair layout).
 * (No reference counterpart.) */
#define FEM_LAYOUT_COLOURS 0
#define FEM_LAYOUT_PAIRS 1
int fem_plan_set_layout(fem_plan *plan, int layout);
int fem_plan_get_layout(const fem_plan *plan, int *layout, int64_t *numPairs, int *numPairColours);
/* Device pointers of the plan's rowp/cols (owned by the plan). */
int fem_plan_device_pattern(const fem_plan *plan, const int **rowp, const int **cols);
/* states/nodeCoords/residual/matEntries are device pointers; residual or
 * matEntries may be NULL to skip that output; matEntries must be 32-byte
 * aligned.  precision: FEM_PRECISION_*. */
int fem_plan_assemble(const fem_plan *plan, const double *states, const double *nodeCoords, double E, double nu,
                      double t, double *residual, double *matEntries, int precision, void *stream,
                      double *elapsedSeconds);
/* Dependency-ordered assembly (opt-in).  With a schedule set, where an assembly
 * runs the fragment kernel (orders 2-4, see FEM_PRECISION_*), fem_plan_assemble
 * runs all colours in ONE persistent launch instead of one launch per colour: the
 * list positions are cut into groups (the elements of one colour within a band of
 * bandElements consecutive element ids) and the groups into tiles of tileElements,
 * dispatched so that each band's later colours follow its earlier ones and its
 * neighbours' within a few bands.  A tile waits (in the kernel, bounded) until the
 * groups whose elements share nodes with its group's, in earlier colours, have
 * finished; every block therefore still receives its contributions in colour
 * order and the result equals the colour launches' bit for bit.  Plans start
 * without a schedule (colour launches, the faster form on large meshes);
 * bandElements = -1 picks a band of about 8 MB of matrix blocks, 0 removes the
 * schedule; tileElements = 0 picks the default (16, order 4: 8).
 * FEM_ERR_UNSUPPORTED for an order-1 plan (row assembly), or when the bands' node
 * ranges overlap too widely (scrambled numbering). */
int fem_plan_set_schedule(fem_plan *plan, int bandElements, int tileElements);
int fem_plan_get_schedule(const fem_plan *plan, int *bandElements, int *tileElements, int *numGroups, int *numTiles);
/* Copies the schedule to host arrays: per tile (numTiles) its first list position,
 * length and group; per group (numGroups) its tile count and, as CSR (depPtr has
 * numGroups + 1 entries), the groups it waits for.  Any pointer may be NULL. */
int fem_plan_get_schedule_tables(const fem_plan *plan, int64_t *tileBegin, int *tileCount, int *tileGroup,
                                 int *groupTiles, int *depPtr, int *deps);
/* Waits for `stream`, then returns (and clears) the number of bounded in-kernel
 * waits of this plan's launches that ran out since the last call: the dependency
 * waits of dependency-ordered launches (each gives up after waitLimitNs, default
 * 0.5 s; the launch then finishes within about one limit) and the tensor-core
 * completion waits of the order-4 MIXED element kernel (2^20 polls).  An assembly
 * with a wait that ran out has invalid results; with elapsedSeconds non-NULL a
 * dependency-ordered fem_plan_assemble checks this itself and returns
 * FEM_ERR_TIMEOUT. */
int fem_plan_wait_status(fem_plan *plan, void *stream, int64_t *timedOutWaits);
/* Failure injection for tests of the bounded waits: waitLimitNs > 0 sets the wait
 * limit; stallGroup >= 0 makes every wait on that group run out (its completion
 * can never be observed), -1 restores normal waits. */
int fem_plan_set_schedule_waits(fem_plan *plan, int64_t waitLimitNs, int stallGroup);

/* fem_plan_assemble with a strain measure (FEM_STRAIN_*; NONLINEAR in FP64 only). */
int fem_plan_assemble_ex(const fem_plan *plan, const double *states, const double *nodeCoords, double E, double nu,
                         double t, double *residual, double *matEntries, int precision, int strainType, void *stream,
                         double *elapsedSeconds);

/* fem_plan_assemble_ex from and to HOST buffers, the copies overlapped with the
 * assembly: the state upload (hostStates -> states) runs in numBands node chunks, the
 * colour launches are split into numBands element bands (element-id ranges) and each
 * band launch starts once the state chunks its nodes need have arrived, and each
 * residual chunk (residual -> hostResidual) is downloaded as soon as the last launch
 * touching its nodes has run.  Launch (band k, colour c) follows every launch of
 * colour c - 1 whose band's node range overlaps band k's, so each block still receives
 * its colours in order: the results equal fem_plan_assemble_ex's bit for bit.  On a
 * mesh numbered along one axis the bands are strips and the copies overlap the
 * assembly; on scrambled numbering the bands overlap each other and it runs serially,
 * with the same result.  hostStates/hostResidual should be pinned (cudaHostAlloc) for
 * the copies to be asynchronous.  The matrix stays on the device (matEntries may be
 * NULL).  Uses two internal streams of the plan, created on the first call; calls on
 * one plan must not overlap.  numBands: 1..256.  (No reference counterpart: the
 * reference driver copies and assembles in sequence, verification/TestKernels.cpp:228-287.) */
int fem_plan_assemble_host(const fem_plan *plan, const double *hostStates, double *states, const double *nodeCoords,
                           double E, double nu, double t, double *hostResidual, double *residual, double *matEntries,
                           int precision, int strainType, int numBands, void *stream, double *elapsedSeconds);

/* ---- batched assembly of many meshes (config: 256 meshes, mixed orders) --------------- */
/* A batch references existing plans (they must outlive it) and assembles all of
 * their meshes with one persistent kernel per (order, colour) -- or, per order,
 * one for all colours (fem_batch_set_ordered) -- whose thread groups pull element
 * tiles from that launch's work queue; the orders run concurrently on internal
 * streams.  Outputs follow fem_plan_assemble (complete overwrite).
 * (No reference counterpart: the reference assembles one mesh per call.) */
typedef struct fem_batch fem_batch;

int fem_batch_create(int numMeshes, fem_plan *const *plans, fem_batch **batch);
int fem_batch_destroy(fem_batch *batch);
/* Device arrays and material of mesh `mesh`; all four arrays are required
 * (vectors 16-byte, matEntries 32-byte aligned).  Rebinding is allowed at any
 * time before the next assemble/replay. */
int fem_batch_bind(fem_batch *batch, int mesh, const double *states, const double *nodeCoords, double E, double nu,
                   double t, double *residual, double *matEntries);
/* Total elements, queue tiles, kernel launches per assembly, device bytes held by the batch. */
int fem_batch_info(const fem_batch *batch, int64_t *totalElements, int64_t *numTiles, int *numLaunches,
                   int64_t *deviceBytes);
/* Tile length per order (index 0..3 = order 1..4), in element batches of the
 * order's kernel shape. */
int fem_batch_get_tiles(const fem_batch *batch, int *tileBatches);
int fem_batch_set_tiles(fem_batch *batch, const int *tileBatches);
/* Kernel variants of a batch, per order and precision.  FEM_KERNEL_DEFAULT is the
 * single-mesh plan path's kernel (batched results then equal the plan's bit for
 * bit); the others trade threads per element and elements per CTA:
 *   ROWS           order 1: row assembly, each block row written once by its warp
 *                  (meshes without row tables take the element kernel)
 *   FRAGMENT_FP64  orders 2-4: two elements per warp in FP64 tensor-core fragments
 *                  (16 threads per element, 8 elements per 4-warp CTA step)
 *   FRAGMENT_BF16X6  order 3, MIXED: the same with the BF16x6 element stiffness
 *   ELEMENT_FP64 / ELEMENT_FP32  every order: the shared-memory element kernel
 *                  (thread groups of 64-128 threads over 1-8 elements, 1-4 groups
 *                  per CTA), FP64 or (MIXED only) FP32 element products.
 *   ELEMENT_TCGEN05  order 4, MIXED: the element kernel with its element stiffness
 *                  as BF16x6 products on the fifth-generation tensor cores (one
 *                  64 x 64 x 32 tcgen05 product per element, FP32 accumulator in
 *                  TMEM); the single-mesh MIXED order-4 path runs it when the
 *                  environment sets FEM_ORDER4_MIXED_STIFFNESS=tcgen05 (read once
 *                  per process), ELEMENT_FP32 otherwise.
 * A MIXED batch may run any FP64 variant: FP64 results are within its bound. */
#define FEM_KERNEL_DEFAULT 0
#define FEM_KERNEL_ROWS 1
#define FEM_KERNEL_FRAGMENT_FP64 2
#define FEM_KERNEL_FRAGMENT_BF16X6 3
#define FEM_KERNEL_ELEMENT_FP64 4
#define FEM_KERNEL_ELEMENT_FP32 5
#define FEM_KERNEL_ELEMENT_TCGEN05 6
/* kernels[4] (orders 1..4) resolved (never DEFAULT) / set (DEFAULT allowed);
 * FEM_ERR_INVALID_ARGUMENT for a variant that cannot serve its order at `precision`. */
int fem_batch_get_kernels(const fem_batch *batch, int precision, int *kernels);
int fem_batch_set_kernels(fem_batch *batch, int precision, const int *kernels);
/* Per order (index 0..3 = order 1..4; order 1 must be 0): 1 runs the order's
 * colours, when its variant is a fragment kernel, as ONE dependency-ordered
 * persistent launch instead of one launch per colour: the tiles of every (mesh,
 * colour) group are dispatched colours outermost, and a tile waits (in the kernel,
 * bounded) until its mesh's previous colour has finished, so every block still
 * receives its contributions in colour order and the result is the same bit for
 * bit.  Batches start with 0; fem_batch_tune chooses per order. */
int fem_batch_set_ordered(fem_batch *batch, const int *ordered);
int fem_batch_get_ordered(const fem_batch *batch, int *ordered);
/* Waits for `stream`, then returns (and clears) the number of bounded in-kernel
 * waits of the batch's dependency-ordered launches that ran out (each gives up
 * after waitLimitNs, default 0.5 s); an assembly with a wait that ran out has
 * invalid results. */
int fem_batch_wait_status(fem_batch *batch, void *stream, int64_t *timedOutWaits);
/* Failure injection for tests of the bounded waits of order `order`'s
 * dependency-ordered launch: waitLimitNs > 0 sets the wait limit; stallGroup >= 0
 * makes every wait on that group (0 = the first mesh's colour 0) run out, -1
 * restores normal waits. */
int fem_batch_set_schedule_waits(fem_batch *batch, int64_t waitLimitNs, int order, int stallGroup);
/* One assembly of every mesh, stream-ordered on `stream`. */
int fem_batch_assemble(fem_batch *batch, int precision, void *stream, double *elapsedSeconds);
/* Autotuner: per order, times the order's launches for every kernel variant the
 * precision allows, every candidate tile length (1, 4, 16, 64, 256 element
 * batches; reps repetitions after a warm-up) and, for the fragment kernels, both
 * launch forms (per colour, dependency-ordered), and keeps the fastest
 * (fem_batch_get_kernels / fem_batch_get_tiles / fem_batch_get_ordered report it).  Replaces the
 * (order, precision) reference tables of hand-tuned elements per block
 * (element/FEKernels.h:1009-1028, 1104-1123). */
int fem_batch_tune(fem_batch *batch, int precision, void *stream, int reps, double *bestSeconds);
/* Captures one complete assembly into a CUDA graph (after one uncaptured warm-up
 * run on `stream`); fem_batch_replay launches it.  Rebinding arrays does not
 * require a new capture (the graph reads the mesh table from device memory);
 * changing tiles does. */
int fem_batch_capture(fem_batch *batch, int precision, void *stream);
int fem_batch_replay(fem_batch *batch, void *stream, double *elapsedSeconds);

/* ---- serving: continuous batching over device-resident meshes ------------------------- */
/* A server keeps client meshes resident (plan, coordinates, state, residual and
 * matrix) within a device-memory budget and assembles submitted requests in
 * waves: whenever one of its eight lanes is free, the pending requests of meshes
 * with at most 2^15 elements (in arrival order, up to 2^17 elements per wave),
 * or, when there are none or the oldest request has waited 10 ms, all pending
 * requests in arrival order (up to maxBatch, and past the first up to 2^21
 * elements) are copied in, assembled by the batched persistent kernels (waves
 * of at most 2^17 elements on a high-priority stream) and their residuals copied
 * back, smallest first, while other lanes may still be running; each request
 * completes as soon as its own residual has arrived.  Host state and residual
 * buffers should be page-locked: a pageable one makes its copy synchronous.
 * (No reference counterpart.) */
typedef struct fem_server fem_server;

int fem_server_create(int64_t budgetBytes, int precision, int maxBatch, fem_server **server);
int fem_server_destroy(fem_server *server);
/* Registers a mesh (host topology and coordinates); FEM_ERR_BUDGET when its
 * device bytes do not fit the remaining budget (retry after a removal). */
int fem_server_add_mesh(fem_server *server, int elementOrder, int numNodes, const int *connPtr, const int *conn,
                        int numElements, const double *nodeCoords, double E, double nu, double t, int *meshId);
int fem_server_remove_mesh(fem_server *server, int meshId);
/* Device pointers of a mesh's resident outputs and pattern (valid until removal). */
int fem_server_mesh_outputs(fem_server *server, int meshId, const double **residual, const double **matEntries,
                            const int **rowp, const int **cols, int64_t *nnzb);
/* One request: hostStates (numNodes*2 doubles, read when the wave is issued) and
 * an optional hostResidual to receive the residual.  One request per mesh may be
 * in flight.  Pinned host buffers let the copies overlap. */
int fem_server_submit(fem_server *server, int meshId, const double *hostStates, double *hostResidual, int64_t *ticket);
/* Waits up to timeoutMs for a ticket; returns its submit-to-completion latency. */
int fem_server_wait(fem_server *server, int64_t ticket, int timeoutMs, double *latencySeconds);
int fem_server_stats(fem_server *server, int64_t *waves, int64_t *completed, int64_t *elements, int64_t *usedBytes,
                     int64_t *budgetBytes);

/* ---- batched drop-in assembly without device allocation --------------------------------- */
/* One mesh in the reference's drop-in format (all arrays are the caller's device
 * memory, laid out as for fem_run_jacobian; residual is required here). */
typedef struct {
  int elementOrder;
  int numElements;
  const int *connPtr;
  const int *conn;
  const double *states;
  const double *nodeCoords;
  double E, nu, t;
  const int *elementBCSRMap;
  double *residual;
  double *matEntries;
} fem_dropin_mesh;

/* Bytes of the library's file-scope device scratch array (the argument table of
 * up to 256 meshes, up to 16384 work-queue tiles and the queue counters). */
#define FEM_STATIC_SCRATCH_BYTES 299008

/* fem_run_jacobian for up to 256 meshes of mixed orders in one batched pass
 * (one persistent launch per order present), for callers that cannot allocate
 * device memory: it calls no cudaMalloc, cudaFree or other allocating routine.
 * What the batched kernel needs besides the caller's arrays lives in a
 * file-scope __device__ array of FEM_STATIC_SCRATCH_BYTES that every GPU using
 * the library holds until the process exits.  The first call on a device looks
 * up that array's device address (make it before any stream capture); the
 * address is cached for the device's context, so the library must be reloaded
 * after cudaDeviceReset.  Calls share the array, so calls that overlap on the
 * GPU race; each call clears the queue counters it uses.  Accumulates into
 * caller-zeroed residual and matEntries like fem_run_jacobian; asynchronous on
 * `stream` except that the mesh table is staged in pageable host memory, whose
 * copy CUDA may start only after the work already queued on `stream` (the call
 * can block the host until then; the staging is free again when it returns).
 * A stream that is being captured is refused (FEM_ERR_UNSUPPORTED): a captured
 * copy would re-read the host staging at every replay.  More than 256 meshes or
 * more work than the tile capacity returns FEM_ERR_UNSUPPORTED.
 * (No counterpart in the reference: it assembles one mesh per call.) */
int fem_run_jacobian_batched_static(int numMeshes, const fem_dropin_mesh *meshes, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FEM_B200_H */
