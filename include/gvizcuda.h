/*
 * gvizcuda.h -- C ABI of libgvizcuda, the B200 (sm_100a) implementation of
 * gviz's force-directed layout step.
 *
 * Plain pointers and sizes only. Every entry point names the reference
 * interface it stands in for (paths inside the Pretz0za/Grapher tree). The
 * gviz-side glue that attaches this library to an existing
 * gvizForceEmbedderState and takes over the "forceEmbedder.step" action is
 * declared in gvizCudaForceEmbedder.h.
 *
 * Layouts:
 *   - vertices are in the embedder's compact order (state->vertices[i] -> i,
 *     include/embedders/gvizForceEmbedder.h:44-46);
 *   - positions / forces are interleaved x0,y0,x1,y1,... FP64, as in
 *     state->positionsScratch (include/embedders/gvizForceEmbedder.h:85-87);
 *   - adjacency is CSR over compact indices, rows in the order the subgraph
 *     neighbour iterator yields them (src/ds/gvizSubgraph.c:466-519);
 *   - a "batch" is several independent graphs concatenated: graph g owns the
 *     vertices [graphOffsets[g], graphOffsets[g+1]) and has its own quadtree,
 *     global speed and stat series.
 *
 * Threading: one handle is driven from one host thread at a time; every
 * handle owns its CUDA stream. Errors are returned as negative codes and
 * latched per handle (gvizCudaForceLastError); nothing aborts the process.
 */
#ifndef GVIZCUDA_H
#define GVIZCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* force models: same values as gvizForceModelKind
 * (include/embedders/gvizForceModel.h:8-11) */
#define GVIZ_CUDA_MODEL_FR 0
#define GVIZ_CUDA_MODEL_LINLOG 1

/* arithmetic of the force walk (positions and speed reductions are FP64 in
 * both): FP32 with Kahan-compensated per-vertex sums, or FP64 with the
 * reference's operation order and no fused multiply-add */
#define GVIZ_CUDA_FP32 0
#define GVIZ_CUDA_FP64 1

/* status codes; -1 and -2 keep the reference's meaning
 * (include/embedders/gvizForceEmbedder.h:161) */
#define GVIZ_CUDA_OK 0
#define GVIZ_CUDA_ERR_ALLOC (-1)      /* device or host allocation failed */
#define GVIZ_CUDA_ERR_DIMENSION (-2)  /* only 2-D layouts are supported */
#define GVIZ_CUDA_ERR_ARG (-3)        /* invalid argument */
#define GVIZ_CUDA_ERR_CUDA (-4)       /* a CUDA runtime call failed */
#define GVIZ_CUDA_ERR_NOT_BEGUN (-5)  /* Run/Step before Begin */
#define GVIZ_CUDA_ERR_NONFINITE (-6)  /* a position was NaN or infinite */
#define GVIZ_CUDA_ERR_DEEP_RUN (-7)   /* > 4096 distinct points share one
                                         depth-32 quadtree cell */
#define GVIZ_CUDA_ERR_NO_DEVICE (-8)  /* no usable CUDA device */
#define GVIZ_CUDA_ERR_LIMIT (-9)      /* size beyond a documented limit */

typedef struct gvizCudaForce gvizCudaForce; /* opaque handle */

/* Graph structure handed to gvizCudaForceCreate. */
typedef struct gvizCudaGraphDesc {
  size_t vertexCount;          /* total vertices over all graphs */
  const uint64_t *rowOffsets;  /* vertexCount + 1 */
  const uint32_t *neighbors;   /* rowOffsets[vertexCount] compact indices */
  const uint64_t *degree;      /* vertexCount, or NULL for the row lengths */
  size_t graphCount;           /* 1 for one layout, > 1 for a batch */
  const uint64_t *graphOffsets;/* graphCount + 1, NULL when graphCount == 1 */
  int32_t model;               /* GVIZ_CUDA_MODEL_* */
  int32_t device;              /* CUDA device ordinal */
} gvizCudaGraphDesc;

/* Configuration, field for field the embedder's
 * (include/embedders/gvizForceEmbedder.h:52-125). */
typedef struct gvizCudaForceParams {
  double edgeLength;        /* FR's k */
  double theta;             /* Barnes-Hut opening threshold (side/distance) */
  uint32_t nodesPerCell;    /* quadtree leaf capacity, 1..256 */
  int32_t barnesHutEnabled; /* 0: exact all-pairs repulsion */
  double gravityK;
  double radiusBase;
  double radiusPerDegree;
  double overlapConstant;
  int32_t preventOverlap;
  int32_t precision;        /* GVIZ_CUDA_FP32 or GVIZ_CUDA_FP64 */
  double jitterTolerance;
  int32_t strictReductions; /* 1: sum swing/traction/magnitudes in vertex
                               order like the reference's serial loops */
  int32_t farField;         /* 0: monopole; 1: learned correction (needs
                               gvizCudaForceSetFarFieldModel) */
  double farGroupSpread;    /* learned correction: when the targets of one
                               warp that accept a cell lie within this
                               fraction of their mean distance to it from
                               their centroid, one model evaluation at the
                               centroid serves them all; 0: one per target */
  int32_t farCellGroups;    /* learned correction: 1 walks the tree once per
                               group of at most 32 targets cut from the tree
                               itself (a cell of <= 32 points whose parent
                               holds more, sibling groups packed together);
                               a cell is accepted for the whole group when
                               it passes the opening test from the group's
                               bounding box and lies outside the group, and
                               one model evaluation at the group's centroid
                               corrects every target's monopole force;
                               0: the per-target walk above */
  int32_t farHubTargets;    /* learned correction: the repulsion of this many
                               heaviest vertices (model mass, ties to the
                               lower id; at most vertexCount) comes from the
                               plain monopole walk at farHubTheta instead, one
                               warp per vertex after the learned walk; 0
                               (default): none. LinLog's force on a vertex
                               scales with its mass, so these carry most of
                               the force-weighted error */
  double farHubTheta;       /* their opening threshold (> 0; default 0.35) */
} gvizCudaForceParams;

/* One step's entries of the five stat series the embedder appends
 * (src/embedders/gvizForceEmbedder.c:484-492). */
typedef struct gvizCudaStepStats {
  double maxDisp;
  double speed;
  double meanAttractive;
  double meanRepulsive;
  double meanGravity;
} gvizCudaStepStats;

/* ---- lifecycle ------------------------------------------------------- */

/* Defaults of gvizForceEmbedderInit (src/embedders/gvizForceEmbedder.c:283-294). */
void gvizCudaForceDefaultParams(gvizCudaForceParams *out);

/* Replaces gvizForceEmbedderInit (src/embedders/gvizForceEmbedder.c:219-325):
 * copies the structure to the device, computes mass from degree per model
 * (src/embedders/gvizForceModel.c:5-8, 31) and sizes every device buffer. */
int gvizCudaForceCreate(gvizCudaForce **out, const gvizCudaGraphDesc *graph);

/* Replaces gvizForceEmbedderRelease (src/embedders/gvizForceEmbedder.c:327-355). */
void gvizCudaForceDestroy(gvizCudaForce *h);

/* Replaces the Configure* / Set*Enabled setters
 * (src/embedders/gvizForceEmbedder.c:357-410); values are taken as given. */
int gvizCudaForceSetParams(gvizCudaForce *h, const gvizCudaForceParams *p);
int gvizCudaForceGetParams(const gvizCudaForce *h, gvizCudaForceParams *p);

/* Positions in compact order (2 * vertexCount doubles). */
int gvizCudaForceSetPositions(gvizCudaForce *h, const double *xy);
int gvizCudaForceGetPositions(gvizCudaForce *h, double *xy);

/* The FA2 part of gvizForceEmbedderBegin (src/embedders/gvizForceEmbedder.c:416-424):
 * speed = 1, efficiency = 1, force history zero, iteration 0, stats cleared. */
int gvizCudaForceBegin(gvizCudaForce *h);

/* Reads / overwrites the FA2 state: structForce (2V, may be NULL) and the
 * per-graph global speed and speed efficiency (graphCount each, may be NULL). */
int gvizCudaForceSetFa2State(gvizCudaForce *h, const double *structForce,
                             const double *speed, const double *efficiency);
int gvizCudaForceGetFa2State(gvizCudaForce *h, double *structForce,
                             double *speed, double *efficiency);

/* ---- stepping -------------------------------------------------------- */

/* Replaces gvizForceEmbedderStep (src/embedders/gvizForceEmbedder.c:445-495)
 * with positions resident on the device. Waits for the step; returns graph
 * 0's maxDisp (negative status on failure) and fills stats[graphCount]. */
double gvizCudaForceStep(gvizCudaForce *h, gvizCudaStepStats *stats);

/* The same step end to end over host memory: copies xy (2V, compact order)
 * to the device, steps, copies the new positions back into xy. This is what
 * the gviz action handler does per invocation. */
double gvizCudaForceStepHost(gvizCudaForce *h, double *xy,
                             gvizCudaStepStats *stats);

/* `steps` steps end to end over host memory, like as many gvizCudaForceStepHost
 * calls: before every step the positions go from xy to the device, after it
 * the new positions come back into xy (2V doubles, compact order), as the
 * reference's Run keeps its embedding in host memory every step
 * (src/embedders/gvizForceEmbedder.c:497-510 around :445-495). The copies of
 * consecutive steps are pipelined in pieces: a piece's upload for the next
 * step starts as soon as its download is back, so the two directions share
 * the link's time. For that overlap xy must be page-locked (cudaHostAlloc or
 * cudaHostRegister); pageable memory gives the same results without it.
 * Waits for the last step; returns graph 0's maxDisp of the last step
 * (negative status on failure, checked after the last step) and fills
 * stats[graphCount] for it. The results are those of `steps` StepHost calls. */
double gvizCudaForceRunHost(gvizCudaForce *h, double *xy, uint32_t steps,
                            gvizCudaStepStats *stats);

/* Enqueues n steps without waiting (replayed from a captured CUDA graph). */
int gvizCudaForceEnqueueSteps(gvizCudaForce *h, uint32_t n);
int gvizCudaForceSynchronize(gvizCudaForce *h);

/* Replaces gvizForceEmbedderRun (src/embedders/gvizForceEmbedder.c:497-510):
 * every graph steps until its maxDisp < epsilon or maxIters rounds ran.
 * rounds[graphCount] (may be NULL) receives each graph's round count. */
int gvizCudaForceRun(gvizCudaForce *h, size_t maxIters, double epsilon,
                     uint64_t *rounds);

/* Stat history of graph g since Begin: up to cap rows of 5 doubles
 * {maxDisp, speed, meanAtt, meanRep, meanGrav}; returns the row count. */
int64_t gvizCudaForceStatHistory(gvizCudaForce *h, uint32_t graph,
                                 double *out, size_t cap);

/* Per-vertex results of the last step in compact order (any may be NULL):
 * the state arrays of include/embedders/gvizForceEmbedder.h:82-108. */
int gvizCudaForceGetForces(gvizCudaForce *h, double *disp, double *structForce,
                           double *attMag, double *repMag, double *swing,
                           double *traction, double *applied);

/* ---- inspection ------------------------------------------------------ */

/* Builds the quadtree on the current positions without stepping and
 * reports each point's leaf as (depth, quadrant path; 2 bits per level,
 * MSB first, digits 1..32 in pathHi, 33..64 in pathLo). Matches the leaves
 * of gvizQuadtreeInit (src/ds/gvizQuadtree.c:200-225) point for point. */
int gvizCudaForceTreeLeaves(gvizCudaForce *h, int32_t *leafDepth,
                            uint64_t *pathHi, uint64_t *pathLo,
                            uint64_t *nodeCount);

/* Compressed-tree nodes of the last build (branching nodes and multi-point
 * leaves): depth, path, mass, centre of mass, point count. Returns count. */
int64_t gvizCudaForceTreeNodes(gvizCudaForce *h, size_t cap, int32_t *depth,
                               uint64_t *pathHi, uint64_t *pathLo,
                               double *mass, double *comX, double *comY,
                               uint64_t *count);

/* FP64 exact repulsion (src/embedders/gvizForceEmbedder.c:104-115) of the
 * listed target vertices against all vertices of their graph, on the GPU:
 * the judge of approximate walks. out: 2 * nTargets. */
int gvizCudaForceExactRepulsion(gvizCudaForce *h, const uint32_t *targets,
                                size_t nTargets, double *out);

/* Repulsion of the current walk configuration (no step taken), for error
 * measurements: out 2V compact order. */
int gvizCudaForceRepulsion(gvizCudaForce *h, double *out);

/* Number of pseudo-body + pair interactions the walk evaluates on the
 * current positions (summed over vertices) and node visits per warp. */
int gvizCudaForceCountInteractions(gvizCudaForce *h, uint64_t *interactions,
                                   uint64_t *warpNodeVisits);

/* With the learned correction on: the MLP rows one force evaluation runs.
 * Per-target walk (farCellGroups 0): shared rows (one per warp and cell,
 * evaluated at the centroid of the warp's accepting targets) and per-target
 * rows, and (laneRowCause[3], may be NULL) why per-target rows were used:
 * fewer than two targets accepted the cell, their spread was too wide, or
 * the cell fails the opening test seen from their centroid. Cell-group walk
 * (farCellGroups 1): groupRows = one row per group and accepted cell,
 * laneRows = 0, and laneRowCause = {node visits of the longest group walk,
 * subtrees walked in place because the stack was full
 * (gvizCudaForceSetWalkStackCap), targets walked over all groups}. Zeros
 * when the correction is off. */
int gvizCudaForceCountFarRows(gvizCudaForce *h, uint64_t *groupRows,
                              uint64_t *laneRows, uint64_t *laneRowCause);

/* Per-kernel device time of the last profiled step (CUDA events on the
 * handle's stream). names: up to cap C strings; ms: up to cap values. */
int gvizCudaForceProfileStep(gvizCudaForce *h, size_t cap, const char **names,
                             double *ms);

/* Device time in ms of n back-to-back steps, measured with CUDA events on
 * the handle's stream around the replays of the captured step. */
int gvizCudaForceTimeSteps(gvizCudaForce *h, uint32_t n, float *ms);

/* Number of this library's kernels one step launches (kernel nodes of the
 * captured step graph for the current parameters). */
int gvizCudaForceStepKernelCount(gvizCudaForce *h);

int gvizCudaForceLastError(const gvizCudaForce *h);
const char *gvizCudaErrorString(int code);

/* Lets a caller supply the CUDA stream (a cudaStream_t) the handle uses. */
int gvizCudaForceSetStream(gvizCudaForce *h, void *stream);

/* ---- learned far-field correction ------------------------------------- */

/* No counterpart in the reference: a 10 -> 64 -> 64 -> 2 MLP (ReLU, BF16
 * weights, FP32 accumulate on tensor cores) that predicts the relative
 * correction of a Barnes-Hut pseudo-body force from the cell's offset,
 * extent, mass and second moments, so a large opening threshold keeps the
 * accuracy of a small one. Weights are MLP_PAD floats in the layout
 * w1t[64][16] (input columns >= 10 unused), b1[64], w2t[64][64], b2[64],
 * w3t[8][64] (rows >= 2 unused), b3[8] (entries >= 2 unused). */
typedef struct gvizCudaMlp gvizCudaMlp;

int gvizCudaMlpCreate(gvizCudaMlp **out, int device, uint64_t seed);
void gvizCudaMlpDestroy(gvizCudaMlp *m);
int gvizCudaMlpParamCount(void);
int gvizCudaMlpSetWeights(gvizCudaMlp *m, const float *w);
int gvizCudaMlpGetWeights(gvizCudaMlp *m, float *w);

/* The kernels of the gradient and of training: 1 (default) the tcgen05
 * path (tiles of 128 samples, one M = 128 MMA per layer with the
 * accumulators in tensor memory, weight gradients accumulated there over a
 * CTA's tiles), 0 the mma.sync path (warp tiles of 32 samples). Both round
 * to BF16 at the same places; results differ by FP32 summation order. */
int gvizCudaMlpSetTrainingKernels(gvizCudaMlp *m, int tcgen05);

/* Gradient (master layout) and value of the weighted mean squared error
 * sum_i W_i |MLP(X_i) - T_i|^2 / sum_i W_i over n samples (X n*10, T n*2,
 * W n or NULL), from the BF16 tensor-core forward/backward kernels. */
int gvizCudaMlpGradient(gvizCudaMlp *m, const float *X, const float *T,
                        const float *W, size_t n, float *grad, float *loss);

/* Adam on the same loss: `epochs` passes in mini-batches of `batch`,
 * shuffled per epoch from `seed`; lossOut[epochs] may be NULL. */
int gvizCudaMlpTrain(gvizCudaMlp *m, const float *X, const float *T,
                     const float *W, size_t n, uint32_t epochs, uint32_t batch,
                     float lr, uint64_t seed, float *lossOut);

/* Batch inference: Y (n*2) from X (n*10). */
int gvizCudaMlpInfer(gvizCudaMlp *m, const float *X, size_t n, float *Y);

/* Uses (m != NULL) or stops using (m == NULL) a trained model in this
 * layout's walk when params.farField is set: a cell is accepted when
 * 2h/|c - v| < theta and it does not contain v, and its monopole force gets
 * the model's correction. */
int gvizCudaForceSetFarFieldModel(gvizCudaForce *h, gvizCudaMlp *m);

/* Training pairs on the current positions at opening threshold theta: for
 * each target vertex and each cell the learned walk accepts, the features
 * (10), the exact relative correction (2, from the cell's points in FP64),
 * the monopole magnitude and the target. Returns the number of pairs found;
 * they are written, ordered by target vertex and then cell, only when cap
 * holds them all (call again with a larger cap otherwise). */
int64_t gvizCudaForceHarvestFarField(gvizCudaForce *h, const uint32_t *targets,
                                     size_t nTargets, double theta,
                                     float *features, float *target,
                                     float *fmono, uint32_t *vertex,
                                     size_t cap);

/* Inspection: the target groups of the learned cell-group walk
 * (params.farCellGroups) built on the current positions as a step builds
 * them: groupOf[V] receives each vertex's group index in [0, *groupCount).
 * The numbering of the groups is not defined; the partition is. */
int gvizCudaForceFarGroups(gvizCudaForce *h, uint32_t *groupOf, uint64_t *groupCount);

/* ---- GRIP force phase -------------------------------------------------- */

/* The refinement round of gviz's GRIP embedder
 * (src/embedders/gvizGRIPEmbedder.c:1289-1334) on the device, 2-D: spring
 * forces (calculateSpringForces :892-934: KK springs to the k nearest on
 * coarse layers; on layer 0 GRIP's FR ops along edges and to the k nearest),
 * the local temperature (updateLocalTemp :870-889), the heat-scaled step,
 * removal of the net translation and rotation (:1106-1252) and the move.
 * The MIS filtration, the placement of a new layer's vertices and the
 * k-nearest search stay with the caller (gviz), which hands each layer over
 * with gvizCudaGripSetLayer. Positions are FP64, indexed by vertex. */
typedef struct gvizCudaGrip gvizCudaGrip; /* opaque handle */

/* gvizGRIPRoundStats (include/embedders/gvizGRIPEmbedder.h), plus the mean
 * heat the reference appends as the "grip.heat" stat series */
typedef struct gvizCudaGripRoundStats {
  double maxDisplacement;
  double meanDisplacement;
  double meanForce;
  double meanHeat;
} gvizCudaGripRoundStats;

/* Graph structure (CSR over vertex ids in gviz's neighbour order, the
 * order gvizSubgraphNeighborIterate yields) and device; positions start at 0. */
int gvizCudaGripCreate(gvizCudaGrip **out, size_t vertexCount, const uint64_t *rowOffsets,
                       const uint32_t *neighbors, int32_t device);
void gvizCudaGripDestroy(gvizCudaGrip *h);

/* Positions, 2 * vertexCount doubles (the embedding's vertex positions). */
int gvizCudaGripSetPositions(gvizCudaGrip *h, const double *xy);
int gvizCudaGripGetPositions(gvizCudaGrip *h, double *xy);

/* Makes `layer` current (gvizGRIPEmbedderBegin / NextStage after placement
 * and updateKNNs, :1010-1069): the active vertices in filtration order and
 * each one's k-nearest list (vertex, graph distance) as CSR over that order;
 * resets the decorators of the active vertices and the "displacement
 * calculated" marks of all vertices as clearDecorators (:936-951) does. */
int gvizCudaGripSetLayer(gvizCudaGrip *h, size_t layer, const uint32_t *active,
                         size_t activeCount, const uint64_t *knnOffsets,
                         const uint32_t *knnVertices, const uint32_t *knnDistances);

/* One round (gvizGRIPEmbedderRefineRound); stats may be NULL. Returns
 * GVIZ_CUDA_ERR_NOT_BEGUN before the first gvizCudaGripSetLayer. */
int gvizCudaGripRefineRound(gvizCudaGrip *h, gvizCudaGripRoundStats *stats);

/* 1: the layer sums (mean displacement, centroid, angular momentum,
 * inertia, stats) in the reference's serial order, so every round is
 * bit-identical to the reference's; 0 (default): chunked, deterministic. */
int gvizCudaGripSetStrictReductions(gvizCudaGrip *h, int32_t strict);

/* Runs `rounds` rounds on the device and times them with CUDA events on
 * the handle's stream: all of them (totalMs) and the force kernel alone
 * (forcesMs, may be NULL). Positions stay on the device. */
int gvizCudaGripTimeRounds(gvizCudaGrip *h, uint32_t rounds, float *totalMs, float *forcesMs);

/* Inspection: per vertex heat, last displacement (2) and previous cosine. */
int gvizCudaGripGetDecorators(gvizCudaGrip *h, double *heat, double *disp, double *oldCos);

/* GRIP's k-nearest lists for a layer (updateKNNs :970-1008 with
 * gvizSearchKNearestScratch, src/algorithms/search/gvizKNearest.c:244-306),
 * on all host threads: per source a breadth-first search over the whole
 * graph in neighbour order recording the first k visible vertices reached
 * (visible NULL: all) with their depth. Lists are packed in source order:
 * offsets[sourceCount + 1]; vertices and distances need sourceCount * k
 * entries. Returns the total entries or a negative code. */
int64_t gvizCudaGripKNearest(size_t vertexCount, const uint64_t *rowOffsets,
                             const uint32_t *neighbors, const uint32_t *sources,
                             size_t sourceCount, const uint8_t *visible, uint32_t k,
                             uint64_t *offsets, uint32_t *vertices, uint32_t *distances);

/* ---- allocation-free speed update ------------------------------------- */

/* No counterpart in the reference. For callers that may not allocate device
 * memory while they run (a per-frame render loop that must not stall on the
 * device allocator, or a host program whose GPU memory belongs to another
 * allocator): the ForceAtlas2 global speed update of one layout, computed
 * from structForce and the previous round's structForce that the caller
 * keeps in device memory. Writes swing_i = m_i |f - f_old| to d_swing (may
 * be NULL) and updates d_speedState = {globalSpeed, speedEfficiency} in place
 * with the rule of updateGlobalSpeed (src/embedders/gvizForceEmbedder.c:140-185).
 * All pointers are device pointers; the work is enqueued on `stream` (a
 * cudaStream_t, NULL for the legacy default stream) and the call returns
 * without waiting.
 * Allocates nothing: its scratch is a 64 KiB array built into the library,
 * which every GPU that loads the library holds until the process exits.
 * Limit: vertexCount <= 4096 * 2048 (8,388,608); larger counts return
 * GVIZ_CUDA_ERR_LIMIT. The first call on each device looks up that array's
 * device address with the device current and keeps it for the life of the
 * process; make that first call before any stream capture, and do not call
 * this entry point on a device after cudaDeviceReset of that device (the
 * kept address belonged to the context the reset destroyed). All calls
 * share the array, so calls that overlap on the GPU (different streams
 * without ordering between them) race. Host threads may make first calls
 * concurrently. For one layout the results are bit-identical to the FP64
 * handle-based step's (the same sums in the same order). */
int gvizCudaFa2SpeedUpdateNoAlloc(const double *d_structForce,
                                  const double *d_oldStructForce,
                                  const double *d_mass, size_t vertexCount,
                                  double jitterTolerance, double *d_swing,
                                  double *d_speedState, void *stream);

/* Picks the FP32 walk's launch shape for this layout by timing it on the
 * current positions: blocks of 64 to 512 threads, a static grid (warp w
 * takes the 32 path-sorted targets of task w) or a persistent one (a grid
 * that fills the GPU once; each warp takes tasks from a device counter until
 * none are left), and, unless the caller set one with
 * gvizCudaForceSetWalkStackCap, the stack entries per warp (128, 256 or 512:
 * a smaller stack takes less shared memory, so more warps are resident).
 * Forces do not depend on block size or schedule; a smaller stack that makes
 * a subtree be walked in place changes the order of that target's sums.
 * Keeps the fastest for later steps; reports it (each output may be NULL;
 * gvizCudaForceGetWalkShape reports the stack). Does nothing for FP64, exact
 * or learned walks. No reference counterpart. */
int gvizCudaForceAutotune(gvizCudaForce *h, uint32_t *threads,
                          int32_t *persistent, float *walkMs);

/* Sets the FP32 walk's launch shape directly: threads per block (a multiple
 * of 32, at most 512) and the persistent schedule (1) or the static one. */
int gvizCudaForceSetWalkShape(gvizCudaForce *h, uint32_t threads, int32_t persistent);

/* The plain FP32 walk's launch shape in use: threads per block, persistent
 * schedule (1) or static, and stack entries per warp. Outputs may be NULL. */
int gvizCudaForceGetWalkShape(const gvizCudaForce *h, uint32_t *threads, int32_t *persistent,
                              uint32_t *stackEntries);

/* The judge of the learned walk (no reference counterpart): the plain
 * Barnes-Hut walk stays both the learned walk's fallback and the judge of
 * its error. A check evaluates, on the current positions, the learned walk
 * as configured and the plain walk at plainTheta, and compares each with
 * exact FP64 all-pairs repulsion on `samples` vertices (a seeded sample,
 * drawn once): error = sqrt(sum |F - F_exact|^2 / sum |F_exact|^2) over the
 * sample. When the learned error is above slack times the plain walk's, the
 * handle turns the learned walk off (farField = 0; GetParams shows it) and
 * later steps take the plain walk. The layout state is not changed.
 * With every > 0 a check runs before every `every`-th step replayed while
 * the learned walk is on (Step, StepHost, EnqueueSteps, Run, TimeSteps;
 * the first one before the next such step); every = 0 checks only on
 * request. Defaults: every 0, samples 4096, plainTheta 0.5, slack 1, seed 1. */
int gvizCudaForceSetFarJudge(gvizCudaForce *h, uint32_t every, uint32_t samples,
                             double plainTheta, double slack, uint64_t seed);

/* One check now (see above); each output may be NULL. fellBack = 1 when this
 * check turned the learned walk off. Errors are 0 when the learned walk is
 * off. Synchronous. */
int gvizCudaForceJudgeFarField(gvizCudaForce *h, double *learnedErr, double *plainErr,
                               int32_t *fellBack);

/* Checks run so far, the last check's errors, and whether any check turned
 * the learned walk off. */
int gvizCudaForceFarJudgeStatus(const gvizCudaForce *h, uint64_t *checks, double *learnedErr,
                                double *plainErr, int32_t *fellBack);

/* The FP32 Barnes-Hut walks (plain and learned cell-group) expand the tree
 * 32 nodes at a time through a per-warp stack of pending nodes in shared
 * memory (512 entries); an opened cell whose children do not fit is walked
 * in place with the stackless preorder walk instead (the same decisions).
 * Sets the stack entries the walks may use, 32 to 512 (0 restores the
 * default: the autotuner's pick for the plain walk, else 512);
 * forces agree up to the order of the per-target sums. A tuning and test
 * knob. No reference counterpart. */
int gvizCudaForceSetWalkStackCap(gvizCudaForce *h, uint32_t entries);

/* ---- checkpoints ------------------------------------------------------ */

/* Lossless checkpoint of a layout (or batch) in progress: positions,
 * structForce, global speed and efficiency, iteration counters and the stat
 * history, as raw bytes with a checksum. gviz's own save
 * (gvizEmbeddedGraphSaveEmbedding, src/embedders/gvizEmbeddedGraph.c:428-448)
 * keeps six decimals and no speed state, so it cannot resume a run; loading
 * this file into a handle of the same graph continues bit for bit as if the
 * run had not stopped. Returns 0, or GVIZ_CUDA_ERR_ARG when the file cannot
 * be written. */
int gvizCudaForceSaveCheckpoint(gvizCudaForce *h, const char *name,
                                const char *filename);

/* Restores a checkpoint into a handle created from the same graph (vertex
 * and graph counts, graph offsets and model must match). restoreParams: 1
 * also restores the configuration saved with it. nameOut (may be NULL)
 * receives the saved name, truncated to nameCap - 1 bytes. Returns 0, or
 * GVIZ_CUDA_ERR_ARG for a file that is missing, damaged (checksum) or from
 * another graph; the handle is unchanged then. */
int gvizCudaForceLoadCheckpoint(gvizCudaForce *h, const char *filename,
                                int restoreParams, char *nameOut, size_t nameCap);

/* Positions in gviz's text embedding format (name line, "count dim", one
 * row per vertex) with 17 significant digits, which
 * gvizEmbeddedGraphLoadEmbedding (src/embedders/gvizEmbeddedGraph.c:450-485)
 * reads back exactly. Vertex i is compact index i (the parent id for a full
 * subgraph). */
int gvizCudaForceSaveEmbeddingText(gvizCudaForce *h, const char *name,
                                   const char *filename);

/* ---- graph files straight to CSR ------------------------------------- */

/* A graph loaded from a file, in the layout's CSR form (library-owned
 * arrays; release with gvizCudaCsrFree). Vertex numbering and neighbour
 * order are those of gviz's loader followed by its subgraph neighbour
 * iterator, so the same file gives the same graph here and in gviz. */
typedef struct gvizCudaCsr {
  size_t vertexCount;
  size_t entryCount;     /* rowOffsets[vertexCount] */
  uint64_t *rowOffsets;  /* vertexCount + 1 */
  uint32_t *neighbors;   /* entryCount */
  int64_t *externalIds;  /* .edges files: each vertex's id in the file */
  int32_t directed;      /* 1: rows hold out-neighbours only */
} gvizCudaCsr;

/* gvizGraphLoadFromEdgesFile (include/utils/graphLoader.h:33-35, Network
 * Repository .edges: "u v [weight]" per line, '%' comments, ids of any
 * base compacted in order of first appearance; skipHeader drops the first
 * data line) without the adjacency-list graph. Unlike gviz's loader, whose
 * id map spans max_id - min_id + 1 entries, sparse huge ids cost nothing
 * extra. Returns 0, or -1 on I/O, parse or allocation failure (out
 * zeroed), or when the graph needs indices beyond 32 bits. */
int gvizCudaLoadEdgesFile(const char *path, int directed, int skipHeader,
                          gvizCudaCsr *out);

/* gvizGraphLoadFromObjFile (include/utils/graphLoader.h:76-89): one vertex
 * per "v" line, edges along each "f" loop (consecutive corners and the
 * closing edge, 1-based or negative relative indices, texture/normal parts
 * ignored, no repeats, no self-loops). Returns 0 or -1 like gviz. */
int gvizCudaLoadObjFile(const char *path, gvizCudaCsr *out);

/* gvizGraphLoadFromGexfFile (include/utils/graphLoader.h:36-61): one vertex
 * per <node> tag in file order (ids matched as strings, the first vertex
 * with an id keeps it), undirected edges in <edge> tag order, with the same
 * scanner and the same failures as gviz's loader (no <node>, a node without
 * an id, an unterminated node or attribute table, a malformed <attvalue>,
 * an edge whose source or target names no node). gviz also builds each
 * vertex's JSON string of label and attribute values; the layout does not
 * use vertex data, so none is built here (externalIds stays NULL).
 * Returns 0 or -1 like gviz. */
int gvizCudaLoadGexfFile(const char *path, gvizCudaCsr *out);

void gvizCudaCsrFree(gvizCudaCsr *csr);

/* ---- host helpers: adjacency and initial placement ------------------- */

/* CSR exactly as gvizGraphAddEdge builds adjacency lists for an undirected
 * graph (src/ds/gvizGraph.c:163-172): edge (a,b) appends b to a's list and
 * a to b's list, in edge order. rowOffsets: V+1; neighbors: 2E. */
int gvizCudaEdgesToCsr(size_t V, const uint32_t *ea, const uint32_t *eb,
                       size_t E, uint64_t *rowOffsets, uint32_t *neighbors);

/* gvizEmbeddedGraphRandomizePositions (src/embedders/gvizEmbeddedGraph.c:406-426)
 * for vertices 0..V-1 in order: the same rand_r draws, x then y. */
void gvizCudaRandomizePositions(double *xy, size_t V, double boxExtent,
                                unsigned seed);

#ifdef __cplusplus
}
#endif

#endif /* GVIZCUDA_H */
