// internal.cuh -- shared definitions of libgvizcuda (B200 / sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gvizcuda.h"

#define GVIZ_NONE 0xFFFFFFFFu
#define GVIZ_KIDS_RUN 0xFFFFFFFEu  // child record of a cell whose children are a run of points
#define GVIZ_LEAF_BIT 0x80000000u
#define GVIZ_MAX_NODES_PER_CELL 256
#define GVIZ_CHUNK 2048          // vertices per reduction chunk
#define GVIZ_FIX_MAX 4096        // largest deep run sorted in shared memory
#define GVIZ_DIR_TABLE 256       // coincident-direction table entries
#define GVIZ_STATS_CAP 4096      // stat rows kept per graph (ring)
#define GVIZ_HEAVY_DEGREE 16     // attraction: warp per vertex above this
#define GVIZ_HUB_DEGREE 4096  // above: split across warps (attraction)
#define GVIZ_HUB_CHUNK 2048   // adjacency entries per hub chunk
#define GVIZ_HOST_PIECES 8    // gvizCudaForceRunHost: pieces of the positions per copy
constexpr uint32_t kWalkDefaultThreads = 128;  // walk block size before autotuning
// The radix sort orders the top 48 bits of the composite (graph, path) key:
// 24 quadtree levels of one graph. Runs equal in those bits and longer than
// the leaf capacity are finished by the shared-memory fix-up sort.
#define GVIZ_SORT_SKIP_BITS 16

// device status bits (OR-ed into ctx->d_status by kernels)
#define GVIZ_ST_NONFINITE 1u
#define GVIZ_ST_DEEP_RUN 2u
#define GVIZ_ST_DEPTH_CAP 4u
#define GVIZ_ST_TREE 8u  // tree invariant broken (guarded, never expected)

#define GVIZ_MAX_CLIMB 256  // binary radix tree depth <= 161 (key bits + 1)

// Per-graph quadtree root: the reference's square root box
// (src/ds/gvizQuadtree.c:165-178) and the depth D at which a node's
// halfSize first drops to <= 1e-9 (an overflow leaf, :134-139).
struct GraphRoot {
  double cx, cy, h0;
  int32_t D;
  int32_t capped;
};

// FP32 walk node, 32 bytes, preorder with skip pointer `next`.
//   info >= 0 : single-point leaf, info = compact vertex index, size = radius
//   info <  0 : cell (branching node or multi-point leaf wrapper),
//               size = (2h/theta)^2, +inf when the cell is never accepted.
// Position / centre of mass as double-single (hi + lo) pairs.
struct __align__(16) NodeF {
  float xh, yh, xl, yl;
  float mass, size;
  int32_t next, info;
};

// FP64 walk node, 48 bytes. size = halfSize h (the reference's test
// 2h/dist < theta), +inf when never accepted; radius for leaves.
struct __align__(16) NodeD {
  double x, y;
  double mass, size;
  int32_t next, info;
  int32_t pad0, pad1;
};

// Side record of a cell (same preorder index as its node record) for the
// learned far-field correction and its training, in the form the features
// use: the second central moments per unit mass (Qxx - Qyy, 2 Qxy,
// Qxx + Qyy, all / M), the halfSize h its opening test uses, the geometric
// centre relative to the centre of mass in units of h, and its points'
// range in path-sorted order.
struct __align__(16) FarCell {
  float qa, qb, tr;
  float h;
  float ox, oy;
  uint32_t s0, s1;
};

struct ChunkStat {
  double a, b, c;  // generic partials
  double pad;
};

struct gvizCudaForce {
  int device = 0;
  cudaStream_t stream = nullptr;
  // attraction depends on positions only: it runs on `side`, forked from
  // and joined back to `stream` around the tree build (null: in order)
  cudaStream_t side = nullptr;
  cudaEvent_t evFork = nullptr, evJoin = nullptr;
  // gvizCudaForceRunHost: the uploads' stream and its events (made at its
  // first call)
  cudaStream_t upload = nullptr;
  cudaEvent_t evDown[GVIZ_HOST_PIECES] = {}, evUp = nullptr;
  bool ownStream = false;
  int model = 0;
  size_t V = 0, E2 = 0, G = 1;
  int gbits = 0;  // bits of the graph id in the composite sort key
  gvizCudaForceParams params{};
  int lastError = 0;
  bool begun = false;
  uint64_t hostIteration = 0;  // steps since Begin (graph 0)

  // host copies
  uint64_t *h_graphOff = nullptr;  // G+1
  double *h_meanDegPlusOne = nullptr;
  uint32_t nChunks = 0;

  // --- structure (device) ---
  uint32_t *d_rowOff = nullptr;  // V+1 (adjacency fits 32 bits)
  uint32_t *d_cols = nullptr;
  uint32_t *d_degree = nullptr;
  double *d_mass = nullptr;
  float *d_massF = nullptr;
  double *d_radius = nullptr;  // 0 when overlap prevention is off
  float *d_radiusF = nullptr;
  uint32_t *d_gid = nullptr;   // per vertex graph id (nullptr when G == 1)
  uint64_t *d_graphOff = nullptr;
  double *d_meanDegPlusOne = nullptr;
  uint32_t *d_chunkBegin = nullptr, *d_chunkEnd = nullptr, *d_chunkGraph = nullptr;
  uint32_t *d_gChunkBegin = nullptr, *d_gChunkEnd = nullptr;
  // attraction work lists: vertices of degree <= GVIZ_HEAVY_DEGREE get a
  // thread, hubs above it a warp
  uint32_t *d_attrLight = nullptr, *d_attrHeavy = nullptr;
  uint32_t nAttrLight = 0, nAttrHeavy = 0;
  // hubs above GVIZ_HUB_DEGREE (power-law graphs reach degrees in the
  // hundreds of thousands): GVIZ_HUB_CHUNK-entry chunks, a warp each, then
  // the chunk partials summed per hub in chunk order
  uint32_t *d_hubV = nullptr, *d_hubFirst = nullptr;  // hubs, nHubs + 1
  uint32_t *d_hubChunkV = nullptr, *d_hubChunkE0 = nullptr, *d_hubChunkE1 = nullptr;
  double2 *d_hubPartial = nullptr;
  uint32_t nHubs = 0, nHubChunks = 0;

  // --- layout state (device) ---
  double2 *d_pos = nullptr;
  double2 *d_sf = nullptr, *d_sfOld = nullptr;
  double2 *d_disp = nullptr, *d_applied = nullptr;
  double *d_att = nullptr, *d_rep = nullptr, *d_swing = nullptr, *d_trac = nullptr;
  float2 *d_attF = nullptr;   // attraction, FP32 path
  double2 *d_attD = nullptr;  // attraction, FP64 path
  double *d_speed = nullptr, *d_eff = nullptr;
  uint32_t *d_active = nullptr;     // per graph: still stepping
  uint32_t *d_anyActive = nullptr;  // 1 while any graph steps
  uint64_t *d_iter = nullptr;       // per graph iteration count
  uint64_t *d_runLeft = nullptr;    // per graph remaining Run rounds
  double *d_runEps = nullptr;
  double *d_stats = nullptr;        // [GVIZ_STATS_CAP][G][5]
  double *d_lastStats = nullptr;    // [G][5], the latest row per graph
  uint64_t *d_counters = nullptr;   // instrumentation counters
  uint32_t *d_walkQueue = nullptr;  // task counter of the persistent walk
  uint2 *d_walkTasks = nullptr;     // walk tasks: first sorted position, targets
  uint32_t nWalkTasks = 0;
  // walk launch shape (gvizCudaForceAutotune): block size, persistent
  // work-queue schedule, and the resident grid for it (0: not measured)
  uint32_t walkThreads = 0;
  bool walkPersistent = false;
  uint32_t walkResident = 0;
  uint32_t walkStackCap = 0;  // FP32 walks: stack entries per warp (0: all)
  uint32_t walkTunedCap = 0;  // plain walk: the autotuner's stack entries (0: all)
  ChunkStat *d_chunkStat = nullptr;
  uint32_t *d_status = nullptr;

  // --- tree build scratch (device) ---
  size_t maxNodes = 0;
  double4 *d_chunkBox = nullptr;
  GraphRoot *d_roots = nullptr;
  uint64_t *d_keyHi = nullptr, *d_keyLo = nullptr;  // per vertex
  uint64_t *d_ck = nullptr, *d_ckAlt = nullptr;     // composite sort keys
  uint32_t *d_idx = nullptr, *d_idxAlt = nullptr;   // sorted vertex ids
  uint64_t *d_sHi = nullptr, *d_sLo = nullptr;      // full keys, sorted order
  uint32_t *d_flag = nullptr, *d_scan = nullptr;    // V-sized
  uint32_t *d_deepRuns = nullptr;
  uint32_t *d_counts = nullptr;  // [0]=runs [1]=deep runs [2]=buckets [3]=nodes
  uint64_t *d_sortState = nullptr;  // radix sort: look-back status, digit counts, tickets
  uint64_t *d_scanState = nullptr;  // scan: ticket and look-back status
  uint64_t *d_bHi = nullptr, *d_bLo = nullptr;
  uint32_t *d_bGid = nullptr, *d_bStart = nullptr;
  uint32_t *d_nLeft = nullptr, *d_nRight = nullptr, *d_nFirst = nullptr,
           *d_nLast = nullptr;
  int32_t *d_nDelta = nullptr;
  uint32_t *d_nCounter = nullptr;
  uint2 *d_upInt = nullptr, *d_upLeaf = nullptr;  // {parent, weight|dead<<31}
  double *d_nM = nullptr, *d_nSX = nullptr, *d_nSY = nullptr;
  uint32_t *d_nCnt = nullptr, *d_nT = nullptr, *d_nFlag = nullptr;
  double *d_bM = nullptr, *d_bSX = nullptr, *d_bSY = nullptr;
  uint32_t *d_bCnt = nullptr, *d_bT = nullptr;
  uint32_t *d_rootNode = nullptr, *d_rootT = nullptr, *d_graphBase = nullptr;
  void *d_nodes = nullptr;  // NodeF or NodeD, maxNodes records
  uint4 *d_kids = nullptr;  // per cell: children's preorder slots (FP32 builds)
  double2 *d_exactPartial = nullptr;  // exact FP32 mode: [exactSplits][V] split sums
  uint32_t exactSplits = 1;
  uint32_t *d_leafDepth = nullptr;  // per vertex (inspection only)

  // forces-only evaluation (no FA2 history update): structForce goes to
  // d_applied and repulsion vectors to repVecOut
  bool forceOnly = false;
  double2 *repVecOut = nullptr;

  // --- learned far-field (mlp.cu) ---
  void *d_mlp = nullptr;
  bool farSide = false;             // build writes FarCell records
  float4 *d_bQ = nullptr, *d_nQ = nullptr;  // second moments (FP32)
  FarCell *d_cells = nullptr;       // maxNodes records
  uint32_t *d_leafPre = nullptr;    // per vertex: preorder index of its leaf
  uint32_t *d_cellCnt = nullptr;    // per cell node: points below it
  uint4 *d_groups = nullptr;        // target groups: preorder [x, y), z points
  uint32_t *d_groupCount = nullptr; // [0] groups written, [1] walk queue
  // hub targets of the learned walk (params.farHubTargets heaviest vertices)
  uint32_t *d_farHubs = nullptr;  // nFarHubs ids, then the walk's hub counter
  double2 *d_farHubOut = nullptr;
  uint32_t nFarHubs = 0;

  // --- judge of the learned walk (api.cu far_judge) ---
  uint32_t judgeEvery = 0;       // steps between automatic checks (0: none)
  uint32_t judgeSamples = 4096;  // sampled target vertices per check
  double judgeTheta = 0.5;       // the plain walk's opening threshold
  double judgeSlack = 1.0;       // learned error may be this times the plain one
  uint64_t judgeSeed = 1;
  uint64_t judgeChecks = 0, judgeNextAt = 0, stepsLaunched = 0;
  double judgeLearned = 0.0, judgePlain = 0.0;
  int32_t judgeFell = 0;
  uint32_t judgeN = 0;             // samples the buffers below hold
  uint32_t *d_judgeIdx = nullptr;  // sampled vertices, ascending
  double2 *d_judgeExact = nullptr, *d_judgeOut = nullptr;  // n; 2n (learned, plain)
  double2 *d_judgeRep = nullptr;   // V: repulsion of one evaluation

  // --- CUDA graph of one step ---
  cudaGraphExec_t stepExec = nullptr;
  bool graphDirty = true;
  int kernelsPerStep = 0;  // kernel nodes in the captured step

  // --- profiling ---
  bool profiling = false;
  int nProf = 0;
  const char *profName[64];
  cudaEvent_t profEv[65];
};

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ void ds_split(double v, float &hi, float &lo) {
  hi = (float)v;
  lo = (float)(v - (double)hi);
}

// coincident direction table (cos, sin of 2*pi*k/256), computed on the host
// with libm and uploaded: identical bits to the oracle's table. One copy per
// translation unit that uses it (no relocatable device code needed).
static __constant__ double c_dirTable[2 * GVIZ_DIR_TABLE];

__device__ __forceinline__ uint64_t gviz_mix64(uint64_t z) {
  z ^= z >> 30;
  z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27;
  z *= 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return z;
}

// Deterministic antisymmetric direction for an exactly coincident pair
// (self, other); replaces the reference's address hash
// (include/core/gvizVec.h:385-394), which no other process can reproduce.
__device__ __forceinline__ void coincident_dir(uint32_t self, uint32_t other,
                                               double &ux, double &uy) {
  uint64_t lo = self < other ? self : other;
  uint64_t hi = self < other ? other : self;
  uint64_t h = gviz_mix64(lo * 0x9e3779b97f4a7c15ULL +
                          gviz_mix64(hi + 0x632be59bd9b4e019ULL));
  int k = (int)(h >> 56);
  ux = c_dirTable[2 * k];
  uy = c_dirTable[2 * k + 1];
  if (self > other) {
    ux = -ux;
    uy = -uy;
  }
}

// ---------------------------------------------------------------------------
// host-side launch helpers
struct EpiArgs;
EpiArgs make_epi(gvizCudaForce *h);  // precise.cu
// ---------------------------------------------------------------------------
// host-side launch helpers (defined in api.cu / sort.cu / tree.cu ...)
// ---------------------------------------------------------------------------

int gviz_check(gvizCudaForce *h, cudaError_t e);
void prof_mark(gvizCudaForce *h, const char *name);

// sort.cu
void radix_sort_pairs(gvizCudaForce *h, uint64_t *keys, uint32_t *vals,
                      uint64_t *keysAlt, uint32_t *valsAlt, size_t n);
void scan_exclusive(gvizCudaForce *h, const uint32_t *in, uint32_t *out,
                    size_t n, uint32_t *total);
size_t sort_state_entries(size_t n);
size_t scan_state_entries(size_t n);

// tree.cu
void enqueue_tree_build(gvizCudaForce *h);
void enqueue_tree_export(gvizCudaForce *h, int32_t *leafDepth);
void enqueue_group_export(gvizCudaForce *h, uint32_t *groupOf);

// mlp.cu
void mlp_free(gvizCudaForce *h);
int far_side_alloc(gvizCudaForce *h);
void far_side_free(gvizCudaForce *h);
int dir_table_upload_forces(const double *t);
int dir_table_upload_precise(const double *t);

// forces.cu (FP32, fused multiply-add on)
void enqueue_attraction_f32(gvizCudaForce *h);
void enqueue_walk_f32(gvizCudaForce *h, uint64_t *counters);
uint32_t walk_resident_blocks(gvizCudaForce *h, uint32_t threads);
uint32_t plain_cap(const gvizCudaForce *h);
void forces_set_smem_limits();
void enqueue_exact_f32(gvizCudaForce *h);
uint32_t exact_splits(size_t V, int sms);

// precise.cu (FP64 + FA2, compiled without fused multiply-add)
void enqueue_attraction_f64(gvizCudaForce *h);
void enqueue_walk_f64(gvizCudaForce *h);
void enqueue_exact_f64(gvizCudaForce *h);
void enqueue_fa2(gvizCudaForce *h);
void enqueue_exact_judge(gvizCudaForce *h, const uint32_t *d_targets,
                         size_t n, double2 *d_out);
