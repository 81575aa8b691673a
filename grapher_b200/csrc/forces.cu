// forces.cu -- FP32 force kernels (compiled with fused multiply-add).
//
//  * k_attr_f32: edge attraction over CSR (src/embedders/gvizForceEmbedder.c:93-100;
//    FR include/core/gvizVec.h:320-334, LinLog :486-499).
//  * k_walk_f32 / k_walk_f32_queue: Barnes-Hut repulsion
//    (src/embedders/gvizForceEmbedder.c:35-74). The 32 lanes of a warp hold 32
//    path-sorted (hence nearby) vertices; the warp expands the union of the
//    nodes they need 32 at a time from a stack of (node, lanes) entries in
//    shared memory, every lane making the reference's own accept / open /
//    pairwise decision for its vertex. An opened cell whose children do not
//    fit the stack is walked in place by the stackless preorder walk.
//  * k_walk_f32_cells / k_walk_f32_far: walks with the learned far-field
//    correction; the first expands the tree the same way with group-wide
//    decisions for tree-cut target groups, the second steps through the
//    warp's union stacklessly with per-target decisions.
//  * k_exact_f32: exact all-pairs repulsion (:104-115), shared-memory tiles,
//    sources split over blockIdx.y (k_exact_combine adds the partials).
//
// Geometry is double-single: a coordinate is hi + lo floats, so a difference
// (ah - bh) + (al - bl) keeps ~FP32 relative accuracy even at |x| ~ 1e3.
// Per-vertex sums are Kahan-compensated FP32 (the walks first add the terms of
// one round, at most 32, in a plain FP32 partial); the epilogue is FP64.
#include <math.h>

#include <algorithm>

#include "epilogue.cuh"
#include "internal.cuh"
#include "mlp.cuh"

int dir_table_upload_forces(const double *t) {
  return cudaMemcpyToSymbol(c_dirTable, t, sizeof(double) * 2 * GVIZ_DIR_TABLE) ==
                 cudaSuccess ? 0 : -1;
}

namespace {

constexpr int kWalkThreads = 128;     // default block size of the walk
constexpr int kWalkMaxThreads = 512;  // largest block size the autotuner tries
constexpr int kAttrThreads = 256;

// 1 / x by the PTX approximate reciprocal (subnormal input and output
// flushed to zero); only the exact kernel's optimistic pass uses it.
__device__ __forceinline__ float rcp_approx_ftz(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

constexpr int kExactThreads = 128;
constexpr int kExactTile = 128;
constexpr int kExactTpt = 4;     // exact mode: targets per thread
constexpr int kExactChunk = 64;  // exact mode: sources per plain partial sum
constexpr uint32_t kInf = 0xffffffffu;

struct Kahan {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const {
    return (double)s - (double)c;
  }
};

struct AttrArgs {
  const uint32_t *rowOff, *cols, *gid, *active, *list;
  const double2 *pos;
  float2 *out;
  float invK;
  uint32_t n;  // entries of list
};

// one attraction term of vertex at p towards q
template <int MODEL>
__device__ __forceinline__ bool attr_term(const double2 p, const double2 q,
                                          float invK, float &tx, float &ty) {
  const float dx = (float)(q.x - p.x);
  const float dy = (float)(q.y - p.y);
  const float dist = sqrtf(dx * dx + dy * dy);
  if (dist < 1e-9f) return false;
  const float s = (MODEL == GVIZ_CUDA_MODEL_FR) ? dist * invK : log1pf(dist) / dist;
  tx = s * dx;
  ty = s * dy;
  return true;
}

// Vertices with at most kHeavyDegree neighbours: one thread each.
template <int MODEL>
__global__ __launch_bounds__(kAttrThreads) void k_attr_f32_light(AttrArgs a) {
  const uint32_t i = blockIdx.x * kAttrThreads + threadIdx.x;
  if (i >= a.n) return;
  const uint32_t v = a.list[i];
  if (a.active && !a.active[a.gid ? a.gid[v] : 0u]) return;
  const double2 p = a.pos[v];
  Kahan kx, ky;
  const uint32_t e1 = a.rowOff[v + 1];
  for (uint32_t e = a.rowOff[v]; e < e1; e++) {
    float tx, ty;
    if (attr_term<MODEL>(p, a.pos[a.cols[e]], a.invK, tx, ty)) {
      kx.add(tx);
      ky.add(ty);
    }
  }
  a.out[v] = make_float2((float)kx.value(), (float)ky.value());
}

// Hubs (scale-free graphs reach degrees in the thousands): one warp each,
// lane-strided Kahan sums combined by a fixed shuffle tree in FP64.
template <int MODEL>
__global__ __launch_bounds__(kAttrThreads) void k_attr_f32_heavy(AttrArgs a) {
  const uint32_t w = (blockIdx.x * kAttrThreads + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (w >= a.n) return;
  const uint32_t v = a.list[w];
  if (a.active && !a.active[a.gid ? a.gid[v] : 0u]) return;
  const double2 p = a.pos[v];
  Kahan kx, ky;
  const uint32_t e1 = a.rowOff[v + 1];
  for (uint32_t e = a.rowOff[v] + lane; e < e1; e += 32) {
    float tx, ty;
    if (attr_term<MODEL>(p, a.pos[a.cols[e]], a.invK, tx, ty)) {
      kx.add(tx);
      ky.add(ty);
    }
  }
  double sx = kx.value(), sy = ky.value();
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
  }
  if (lane == 0) a.out[v] = make_float2((float)sx, (float)sy);
}

// Hubs above GVIZ_HUB_DEGREE: one warp per GVIZ_HUB_CHUNK-entry chunk of
// the hub's adjacency, each writing an FP64 partial ...
struct HubArgs {
  const uint32_t *rowOff, *cols, *gid, *active;
  const uint32_t *chunkV, *chunkE0, *chunkE1, *hubV, *hubFirst;
  const double2 *pos;
  double2 *partial;
  float2 *out;
  float invK;
  uint32_t nChunks, nHubs;
};

template <int MODEL>
__global__ __launch_bounds__(kAttrThreads) void k_attr_f32_hub_chunks(HubArgs a) {
  const uint32_t w = (blockIdx.x * kAttrThreads + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (w >= a.nChunks) return;
  const uint32_t v = a.chunkV[w];
  if (a.active && !a.active[a.gid ? a.gid[v] : 0u]) return;
  const double2 p = a.pos[v];
  Kahan kx, ky;
  const uint32_t e1 = a.chunkE1[w];
  for (uint32_t e = a.chunkE0[w] + lane; e < e1; e += 32) {
    float tx, ty;
    if (attr_term<MODEL>(p, a.pos[a.cols[e]], a.invK, tx, ty)) {
      kx.add(tx);
      ky.add(ty);
    }
  }
  double sx = kx.value(), sy = ky.value();
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
  }
  if (lane == 0) a.partial[w] = make_double2(sx, sy);
}

// ... then each hub's partials summed in chunk order (deterministic).
__global__ __launch_bounds__(kAttrThreads) void k_attr_hub_sum(HubArgs a) {
  const uint32_t i = blockIdx.x * kAttrThreads + threadIdx.x;
  if (i >= a.nHubs) return;
  const uint32_t v = a.hubV[i];
  if (a.active && !a.active[a.gid ? a.gid[v] : 0u]) return;
  double sx = 0.0, sy = 0.0;
  for (uint32_t c = a.hubFirst[i]; c < a.hubFirst[i + 1]; c++) {
    sx += a.partial[c].x;
    sy += a.partial[c].y;
  }
  a.out[v] = make_float2((float)sx, (float)sy);
}

struct WalkArgs {
  const NodeF *nodes;
  const uint4 *kids;  // per cell: children's preorder slots (tree build)
  const uint32_t *idx, *gid, *active, *graphBase, *rootT;
  const double2 *pos;
  const float *massF, *radiusF;
  const float2 *attF;
  EpiArgs epi;
  float num;     // FR: k^2
  uint32_t maxNodes;
  float overlapC;
  uint32_t V;
  unsigned long long *counters;  // [0] interactions, [1] warp node visits
  uint32_t *queue;               // next task of the persistent schedule
  uint32_t stackCap;             // stack entries per warp in use
  const uint2 *tasks;            // plain walk tasks: first sorted position, targets
  uint32_t nTasks;
};

// One pair or pseudo-body term of FR / LinLog repulsion
// (include/core/gvizVec.h:404-428, 552-578; FR mass truncation
// src/embedders/gvizForceModel.c:20).
template <int MODEL, bool OVERLAP>
__device__ __forceinline__ void rep_term(float dx, float dy, float d2,
                                         float mv, float mo, float radiusSum,
                                         float num, float C, uint32_t self,
                                         uint32_t other, float &fx, float &fy) {
  const float numer = (MODEL == GVIZ_CUDA_MODEL_FR) ? num : mv * mo;
  const float mult = (MODEL == GVIZ_CUDA_MODEL_FR) ? truncf(mo) : 1.0f;
  if (d2 > 0.0f) {
    if (OVERLAP) {
      const float inv = rsqrtf(d2);
      const float dist = d2 * inv;
      const float gap = dist - radiusSum;
      const float mag = gap > 0.0f ? __fdividef(numer, gap) : numer * C;
      const float s = mag * inv * mult;
      fx = __fmul_rn(-s, dx);  // never fused into the caller's sums
      fy = __fmul_rn(-s, dy);
    } else {
      const float s = __fdividef(numer, d2) * mult;
      fx = __fmul_rn(-s, dx);  // never fused into the caller's sums
      fy = __fmul_rn(-s, dy);
    }
  } else {
    double ux, uy;
    coincident_dir(self, other, ux, uy);
    const float mag = numer * C * mult;
    fx = __fmul_rn(-mag, (float)ux);
    fy = __fmul_rn(-mag, (float)uy);
  }
}

// rep_term for d2 > 0: the same arithmetic, without the coincident branch,
// so the common case compiles to straight-line predicated code.
template <int MODEL, bool OVERLAP>
__device__ __forceinline__ void rep_term_apart(float dx, float dy, float d2, float mv,
                                               float mo, float radiusSum, float num,
                                               float C, float &fx, float &fy) {
  const float numer = (MODEL == GVIZ_CUDA_MODEL_FR) ? num : mv * mo;
  const float mult = (MODEL == GVIZ_CUDA_MODEL_FR) ? truncf(mo) : 1.0f;
  if (OVERLAP) {
    const float inv = rsqrtf(d2);
    const float dist = d2 * inv;
    const float gap = dist - radiusSum;
    const float mag = gap > 0.0f ? __fdividef(numer, gap) : numer * C;
    const float s = mag * inv * mult;
    fx = __fmul_rn(-s, dx);  // never fused into the caller's sums
    fy = __fmul_rn(-s, dy);
  } else {
    const float s = __fdividef(numer, d2) * mult;
    fx = __fmul_rn(-s, dx);  // never fused into the caller's sums
    fy = __fmul_rn(-s, dy);
  }
}

// One walk task: the 32 path-sorted targets starting at sorted position
// 32 * task, one per lane, each making the reference's own decisions
// (bhAccumulateRepulsion, src/embedders/gvizForceEmbedder.c:35-74): empty
// node skipped; point: pair term unless it is the target; cell: accepted
// when 2h/|com - v| < theta, else opened. The warp expands the union of
// the nodes its lanes need 32 at a time: a pending entry is a node and the
// lanes whose walks reach it (they opened every ancestor); each round every
// lane pops one entry and loads its node (32 independent loads), the
// records go to shared memory, and then every lane tests each of the round's
// nodes for its own target if it is among that node's lanes. An opened node
// pushes its children (slots from the tree build's child records) with the
// lanes that opened it. A push that would overflow the stack is walked in
// place with the stackless union walk below (the same decisions).
constexpr int kPlainStack = 512;  // largest stack: pending (node, lanes) entries per warp

// A warp's region of the plain walk's dynamic shared memory: the round's 32
// node records (1 KiB), then a stack of stackCap entries; the region's
// size follows the stack cap, so a smaller stack leaves room for more
// resident warps.
struct PlainWarpSmem {
  float4 (*rec)[2];  // the round's node records
  uint2 *st;         // pending entries: node, lanes
};

__host__ __device__ constexpr uint32_t plain_warp_bytes(uint32_t cap) {
  return 32u * 2u * 16u + ((cap * 8u + 15u) & ~15u);
}

__device__ __forceinline__ PlainWarpSmem plain_warp_smem(unsigned char *dyn, uint32_t cap) {
  unsigned char *base = dyn + (size_t)(threadIdx.x >> 5) * plain_warp_bytes(cap);
  PlainWarpSmem q;
  q.rec = reinterpret_cast<float4(*)[2]>(base);
  q.st = reinterpret_cast<uint2 *>(base + 32 * 2 * 16);
  return q;
}

struct PlainTarget {
  uint32_t v;
  bool act;
  float vxh, vxl, vyh, vyl, mv, rv;
};

// The reference's decision for one node and this lane's target: adds the
// term of a point or an accepted cell; returns true when the cell is opened.
template <int MODEL, bool OVERLAP>
__device__ __forceinline__ bool plain_visit(const WalkArgs &a, const PlainTarget &t, bool in,
                                            float4 n0, float4 n1, float &px, float &py,
                                            unsigned long long &nInter) {
  const float nmass = n1.x, nsize = n1.y;
  const int32_t ninfo = __float_as_int(n1.w);
  const float dx = (n0.x - t.vxh) + (n0.z - t.vxl);
  const float dy = (n0.y - t.vyh) + (n0.w - t.vyl);
  const float d2 = dx * dx + dy * dy;
  const bool isLeaf = ninfo >= 0;
  const bool massOk = nmass != 0.0f;
  const bool accept = !isLeaf && nsize < d2;
  const bool doForce = in && massOk && (isLeaf ? ((uint32_t)ninfo != t.v) : accept);
  // coincident points are rare: one vote keeps their branch off the
  // common path, which stays straight-line
  if (__any_sync(0xffffffffu, doForce && !(d2 > 0.0f))) {
    if (doForce) {
      float fx, fy;
      rep_term<MODEL, OVERLAP>(dx, dy, d2, t.mv, nmass, t.rv + (isLeaf ? nsize : 0.0f), a.num,
                               a.overlapC, t.v, isLeaf ? (uint32_t)ninfo : t.v, fx, fy);
      px += fx;
      py += fy;
    }
  } else if (doForce) {
    float fx, fy;
    rep_term_apart<MODEL, OVERLAP>(dx, dy, d2, t.mv, nmass, t.rv + (isLeaf ? nsize : 0.0f),
                                   a.num, a.overlapC, fx, fy);
    px += fx;
    py += fy;
  }
  nInter += doForce ? 1ull : 0ull;
  return in && massOk && !isLeaf && !accept;
}

// plain_visit without the coincidence vote: the term of a point or accepted
// cell on the straight-line path (a coincident point gives a term that is
// not finite; the caller then redoes the round with plain_visit).
template <int MODEL, bool OVERLAP>
__device__ __forceinline__ bool plain_visit_fast(const WalkArgs &a, const PlainTarget &t, bool in,
                                                 float4 n0, float4 n1, float &px, float &py) {
  const float nmass = n1.x, nsize = n1.y;
  const int32_t ninfo = __float_as_int(n1.w);
  const float dx = (n0.x - t.vxh) + (n0.z - t.vxl);
  const float dy = (n0.y - t.vyh) + (n0.w - t.vyl);
  const float d2 = dx * dx + dy * dy;
  const bool isLeaf = ninfo >= 0;
  const bool massOk = nmass != 0.0f;
  const bool accept = !isLeaf && nsize < d2;
  const bool doForce = in && massOk && (isLeaf ? ((uint32_t)ninfo != t.v) : accept);
  if (doForce) {
    float fx, fy;
    rep_term_apart<MODEL, OVERLAP>(dx, dy, d2, t.mv, nmass, t.rv + (isLeaf ? nsize : 0.0f),
                                   a.num, a.overlapC, fx, fy);
    px += fx;
    py += fy;
  }
  return in && massOk && !isLeaf && !accept;
}

// The stackless union walk of the preorder range [lo, hi) for the lanes in
// `lanes`: the warp steps through the union of the nodes they need, each
// lane's next node is cur + 1 (opened) or the node's skip pointer, the warp
// moves to the minimum.
template <int MODEL, bool OVERLAP>
__device__ void plain_walk_range(const WalkArgs &a, const PlainTarget &t, uint32_t lanes,
                                 uint32_t lo, uint32_t hi, Kahan &kx, Kahan &ky,
                                 unsigned long long &nInter, unsigned long long &nVisit) {
  const uint32_t lane = threadIdx.x & 31u;
  const bool mine = (lanes >> lane) & 1u;
  uint32_t resume = mine ? lo : kInf;
  uint32_t cur = __reduce_min_sync(0xffffffffu, resume < hi ? resume : kInf);
  float px = 0.f, py = 0.f;
  uint32_t run = 0;
  while (cur != kInf) {
    const float4 n0 = __ldg(reinterpret_cast<const float4 *>(a.nodes + cur));
    const float4 n1 = __ldg(reinterpret_cast<const float4 *>(a.nodes + cur) + 1);
    const bool in = mine && cur == resume;
    const bool open = plain_visit<MODEL, OVERLAP>(a, t, in, n0, n1, px, py, nInter);
    if (in) resume = open ? cur + 1u : max((uint32_t)__float_as_int(n1.z), cur + 1u);
    nVisit++;
    if (++run == 32u) {  // the cascade of the round-based walk: 32 terms, then Kahan
      kx.add(px);
      ky.add(py);
      px = py = 0.f;
      run = 0;
    }
    cur = __reduce_min_sync(0xffffffffu, resume < hi ? resume : kInf);
  }
  kx.add(px);
  ky.add(py);
}

template <int MODEL, bool OVERLAP, bool COUNT>
__device__ __forceinline__ void walk_task(const WalkArgs &a, uint32_t task, const PlainWarpSmem &q) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t below = (1u << lane) - 1u;
  // a task's targets all belong to one graph (tasks are cut per graph): the
  // order of each target's sums depends only on its graph's layout
  const uint2 tk = a.tasks[task];
  const uint32_t s = tk.x + lane;
  const bool valid = lane < tk.y && s < a.V;
  PlainTarget t;
  t.v = valid ? a.idx[s] : 0u;
  const uint32_t g = (valid && a.gid) ? a.gid[t.v] : 0u;
  t.act = valid && (a.active == nullptr || a.active[g] != 0u);
  uint32_t root = 0, myEnd = 0;
  if (t.act) {
    root = a.graphBase[g];
    myEnd = min(root + a.rootT[g], a.maxNodes);
  }
  t.vxh = t.vxl = t.vyh = t.vyl = t.mv = t.rv = 0.f;
  if (t.act) {
    const double2 p = a.pos[t.v];
    ds_split(p.x, t.vxh, t.vxl);
    ds_split(p.y, t.vyh, t.vyl);
    t.mv = a.massF[t.v];
    if (OVERLAP) t.rv = a.radiusF[t.v];
  }
  Kahan kx, ky;
  unsigned long long nInter = 0, nVisit = 0, nSerial = 0;
  // the first entries: each distinct root among the lanes, with its lanes
  const uint32_t key = (t.act && root < myEnd) ? root : kInf;
  const uint32_t same = __match_any_sync(0xffffffffu, key);
  const bool leader = key != kInf && (uint32_t)(__ffs(same) - 1) == lane;
  const uint32_t bl = __ballot_sync(0xffffffffu, leader);
  if (leader) q.st[__popc(bl & below)] = make_uint2(root, same);
  uint32_t top = __popc(bl);
  __syncwarp();
  while (top > 0u) {
    const uint32_t n = min(top, 32u);
    const bool mine = lane < n;
    const uint2 e = mine ? q.st[top - n + lane] : make_uint2(0u, 0u);
    top -= n;
    float4 n0 = make_float4(0.f, 0.f, 0.f, 0.f), n1 = n0;
    uint4 kd = make_uint4(GVIZ_NONE, GVIZ_NONE, GVIZ_NONE, GVIZ_NONE);
    if (mine) {
      n0 = __ldg(reinterpret_cast<const float4 *>(a.nodes + e.x));
      n1 = __ldg(reinterpret_cast<const float4 *>(a.nodes + e.x) + 1);
      kd = __ldg(a.kids + e.x);  // read for every node; used only when it is opened
    }
    // the graph's end for the entry's lanes (they share one graph)
    const uint32_t entryEnd = __shfl_sync(0xffffffffu, myEnd, mine ? __ffs(e.y) - 1 : 0);
    __syncwarp();  // popped, and last round's records read, before the writes below
    if (mine) {
      q.rec[lane][0] = n0;
      q.rec[lane][1] = n1;
    }
    __syncwarp();
    if (COUNT) nVisit += n;
    // the round's terms in a plain FP32 partial, which then joins the
    // target's Kahan-compensated sum (cascade summation, <= 32 terms a run)
    uint32_t myOpen = 0;
    float px = 0.f, py = 0.f;
    if (COUNT) {  // instrumented: the guarded visits, counting terms
      for (uint32_t j = 0; j < n; j++) {
        const uint32_t lanes = __shfl_sync(0xffffffffu, e.y, j);
        const bool open = plain_visit<MODEL, OVERLAP>(a, t, (lanes >> lane) & 1u, q.rec[j][0],
                                                      q.rec[j][1], px, py, nInter);
        const uint32_t ob = __ballot_sync(0xffffffffu, open);
        if (lane == j) myOpen = ob;
      }
    } else {
      for (uint32_t j = 0; j < n; j++) {
        const uint32_t lanes = __shfl_sync(0xffffffffu, e.y, j);
        const bool open = plain_visit_fast<MODEL, OVERLAP>(a, t, (lanes >> lane) & 1u, q.rec[j][0],
                                                           q.rec[j][1], px, py);
        const uint32_t ob = __ballot_sync(0xffffffffu, open);
        if (lane == j) myOpen = ob;
      }
      // a coincident point in the round: the round again on the guarded path
      // (the same decisions; the open masks above stand)
      if (__any_sync(0xffffffffu, !(isfinite(px) && isfinite(py)))) {
        px = py = 0.f;
        for (uint32_t j = 0; j < n; j++) {
          const uint32_t lanes = __shfl_sync(0xffffffffu, e.y, j);
          plain_visit<MODEL, OVERLAP>(a, t, (lanes >> lane) & 1u, q.rec[j][0], q.rec[j][1], px,
                                      py, nInter);
        }
      }
    }
    kx.add(px);
    ky.add(py);
    // opened nodes push their children (inside the graph's subtree) with the
    // lanes that opened them, in lane order, while they fit
    uint32_t nk = 0;
    if (myOpen) {
      if (kd.y == GVIZ_KIDS_RUN) {
        nk = (kd.x > e.x && kd.x < entryEnd) ? min(kd.z, entryEnd - kd.x) : 0u;
        nk = min(nk, a.stackCap + 1u);  // a longer run never fits
      } else {
        kd.x = (kd.x > e.x && kd.x < entryEnd) ? kd.x : GVIZ_NONE;
        kd.y = (kd.y > e.x && kd.y < entryEnd) ? kd.y : GVIZ_NONE;
        kd.z = (kd.z > e.x && kd.z < entryEnd) ? kd.z : GVIZ_NONE;
        kd.w = (kd.w > e.x && kd.w < entryEnd) ? kd.w : GVIZ_NONE;
        nk = (uint32_t)(kd.x != GVIZ_NONE) + (uint32_t)(kd.y != GVIZ_NONE) +
             (uint32_t)(kd.z != GVIZ_NONE) + (uint32_t)(kd.w != GVIZ_NONE);
      }
    }
    uint32_t incl = nk;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    const bool fits = top + incl <= a.stackCap;
    if (myOpen && fits) {
      const uint32_t base = top + incl - nk;
      if (kd.y == GVIZ_KIDS_RUN) {
        for (uint32_t i = 0; i < nk; i++) q.st[base + i] = make_uint2(kd.x + i, myOpen);
      } else {
        uint32_t w = base;
        if (kd.x != GVIZ_NONE) q.st[w++] = make_uint2(kd.x, myOpen);
        if (kd.y != GVIZ_NONE) q.st[w++] = make_uint2(kd.y, myOpen);
        if (kd.z != GVIZ_NONE) q.st[w++] = make_uint2(kd.z, myOpen);
        if (kd.w != GVIZ_NONE) q.st[w++] = make_uint2(kd.w, myOpen);
      }
    }
    top += __reduce_max_sync(0xffffffffu, fits ? incl : 0u);
    // subtrees that did not fit, walked in place
    uint32_t bS = __ballot_sync(0xffffffffu, myOpen != 0u && !fits);
    if (COUNT) nSerial += __popc(bS);
    while (bS) {
      const int l = __ffs(bS) - 1;
      bS &= bS - 1u;
      const uint32_t lanes = __shfl_sync(0xffffffffu, myOpen, l);
      const uint32_t lo = __shfl_sync(0xffffffffu, e.x, l) + 1u;
      const uint32_t hi = __shfl_sync(
          0xffffffffu, min(max((uint32_t)__float_as_int(n1.z), e.x + 1u), entryEnd), l);
      plain_walk_range<MODEL, OVERLAP>(a, t, lanes, lo, hi, kx, ky, nInter, nVisit);
    }
    __syncwarp();
  }
  if (COUNT) {
    atomicAdd(a.counters, nInter);
    if (lane == 0) {
      atomicAdd(a.counters + 1, nVisit);
      atomicAdd(a.counters + 5, nSerial);
    }
  }
  if (!t.act) return;
  const float2 at = a.attF[t.v];
  force_epilogue(a.epi, t.v, (double)at.x, (double)at.y, kx.value(), ky.value());
}

// Static schedule: warp w of the grid takes task w.
template <int MODEL, bool OVERLAP, bool COUNT>
__global__ __launch_bounds__(kWalkMaxThreads) void k_walk_f32(WalkArgs a) {
  extern __shared__ __align__(16) unsigned char plainDyn[];
  const PlainWarpSmem q = plain_warp_smem(plainDyn, a.stackCap);
  const uint32_t task = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (task >= a.nTasks) return;  // the whole warp
  walk_task<MODEL, OVERLAP, COUNT>(a, task, q);
}

// Persistent schedule: a grid sized to fill the GPU once; each warp takes
// the next task from a device counter (reset before every launch) until
// the queue is empty, so warps that drew cheap tasks take more of them.
template <int MODEL, bool OVERLAP, bool COUNT>
__global__ __launch_bounds__(kWalkMaxThreads) void k_walk_f32_queue(WalkArgs a) {
  extern __shared__ __align__(16) unsigned char plainDyn[];
  const PlainWarpSmem q = plain_warp_smem(plainDyn, a.stackCap);
  for (;;) {
    uint32_t t = 0;
    if ((threadIdx.x & 31u) == 0u) t = atomicAdd(a.queue, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= a.nTasks) return;
    walk_task<MODEL, OVERLAP, COUNT>(a, t, q);
  }
}

// ---------------------------------------------------------------------------
// The learned walk: as k_walk_f32, with two changes that define the learned
// method (it has no reference counterpart): a cell containing the target is
// never accepted, and every accepted cell's monopole force F gets the MLP's
// correction p1 F + p2 rot90(F) (p = s^2 MLP(features), s = h/d, is the
// relative correction in the frame of F). The MLP runs on the tensor cores over 16-row tiles queued per warp
// in shared memory. The accepting lanes of a cell share a row where their
// targets are close together compared with their distance to it:
//   shared row - lanes within farGroupSpread * |c - g| of the warp's target
//                centroid g (the cell must pass the opening test from g)
//                share one row with the features seen from g; each keeps
//                its own F for it;
//   lane row   - one row per remaining accepting lane.
// One feature pass serves both kinds. Rows are applied in queue order, so
// the sums are deterministic. (Nearly every warp iteration accepts some
// cell, so the per-iteration bookkeeping, not the tensor-core work, sets
// the cost; finer groups, e.g. per quarter-warp, cut rows but cost more.)
// ---------------------------------------------------------------------------

constexpr int kFarThreads = 128;
constexpr int kFarTile = 16;
constexpr int kFarLaneCap = 48;  // a tile plus one warp's worth of overflow

struct FarArgs {
  WalkArgs w;
  const FarCell *cells;
  const uint32_t *leafPre;
  const MlpDev *mlp;
  float spread2;  // farGroupSpread^2
};

struct __align__(16) FarWarpSmem {
  __nv_bfloat16 gx[kFarTile * MLP_XS];     // shared rows
  __nv_bfloat16 lx[kFarLaneCap * MLP_XS];  // lane rows
  float2 gF[kFarTile][32];                 // each lane's F in each shared row
  float2 lF[kFarLaneCap];                  // the owner's F of each lane row
  float2 out[kFarTile];
};

__device__ __forceinline__ void far_put_row(__nv_bfloat16 *row, const float *f) {
  uint4 lo, hi;
  lo.x = pack_bf16(f[0], f[1]);
  lo.y = pack_bf16(f[2], f[3]);
  lo.z = pack_bf16(f[4], f[5]);
  lo.w = pack_bf16(f[6], f[7]);
  hi.x = pack_bf16(f[8], f[9]);
  hi.y = hi.z = hi.w = 0u;
  reinterpret_cast<uint4 *>(row)[0] = lo;
  reinterpret_cast<uint4 *>(row)[1] = hi;
}

__device__ __forceinline__ void far_apply(float2 p, float2 F, float &cx, float &cy) {
  cx += p.x * F.x - p.y * F.y;
  cy += p.x * F.y + p.y * F.x;
}

// sum over the aligned group of `width` lanes (16, 8, ...: xor offsets below
// width); the same bits in every lane of the group
template <int WIDTH>
__device__ __forceinline__ double group_sum_d(double x) {
#pragma unroll
  for (int o = WIDTH / 2; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// centroid (double-single) of the active lanes of an aligned lane group and
// this lane's squared distance to it (INFINITY when inactive)
template <int WIDTH, bool RADIUS>
__device__ __forceinline__ void group_centroid(bool act, double2 p, float vxh, float vxl,
                                               float vyh, float vyl, float rv, float &gxh,
                                               float &gxl, float &gyh, float &gyl,
                                               float &r2, float &grv) {
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t grp = WIDTH == 32 ? 0xffffffffu : (((1u << WIDTH) - 1u) << (lane & ~(WIDTH - 1u)));
  const int na = __popc(__ballot_sync(0xffffffffu, act) & grp);
  const double inv = na > 0 ? 1.0 / (double)na : 0.0;
  ds_split(group_sum_d<WIDTH>(act ? p.x : 0.0) * inv, gxh, gxl);
  ds_split(group_sum_d<WIDTH>(act ? p.y : 0.0) * inv, gyh, gyl);
  grv = RADIUS ? (float)(group_sum_d<WIDTH>(act ? (double)rv : 0.0) * inv) : 0.f;
  r2 = INFINITY;
  if (act) {
    const float ex = (vxh - gxh) + (vxl - gxl), ey = (vyh - gyh) + (vyl - gyl);
    r2 = ex * ex + ey * ey;
  }
}

template <int MODEL, bool OVERLAP, bool COUNT>
__global__ __launch_bounds__(kFarThreads, 5) void k_walk_f32_far(FarArgs fa) {
  __shared__ MlpSmem W;
  __shared__ FarWarpSmem Q[kFarThreads / 32];
  mlp_stage(W, fa.mlp);
  __syncthreads();
  const WalkArgs &a = fa.w;
  FarWarpSmem &q = Q[threadIdx.x >> 5];
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t s = ((blockIdx.x * kFarThreads + threadIdx.x) >> 5) * 32u + lane;
  const bool valid = s < a.V;
  const uint32_t v = valid ? a.idx[s] : 0u;
  const uint32_t g = (valid && a.gid) ? a.gid[v] : 0u;
  const bool act = valid && (a.active == nullptr || a.active[g] != 0u);
  uint32_t resume = 0, myEnd = 0, myLeaf = 0;
  float vxh = 0.f, vxl = 0.f, vyh = 0.f, vyl = 0.f, mv = 0.f, rv = 0.f;
  double2 pv = make_double2(0.0, 0.0);
  if (act) {
    resume = a.graphBase[g];
    myEnd = min(resume + a.rootT[g], a.maxNodes);
    myLeaf = fa.leafPre[v];
    pv = a.pos[v];
    ds_split(pv.x, vxh, vxl);
    ds_split(pv.y, vyh, vyl);
    mv = a.massF[v];
    if (OVERLAP) rv = a.radiusF[v];
  }
  // the warp's target centroid
  float wxh, wxl, wyh, wyl, wr2, wrv;
  group_centroid<32, OVERLAP>(act, pv, vxh, vxl, vyh, vyl, rv, wxh, wxl, wyh, wyl, wr2, wrv);
  const float spread2 = fa.spread2;
  const bool grouping = spread2 > 0.0f;
  Kahan kx, ky;
  float corrx = 0.f, corry = 0.f;
  int qg = 0, ql = 0;  // warp-uniform queue lengths
  uint64_t mine = 0;   // this lane's slots in the lane queue
  unsigned long long nInter = 0, nVisit = 0, nGroup = 0, nLane = 0, nEvent = 0;
  unsigned long long nWhy[3] = {0, 0, 0};
  uint32_t nxt = resume < myEnd ? resume : kInf;
  uint32_t cur = __reduce_min_sync(0xffffffffu, nxt);
  while (cur != kInf) {
    const float4 n0 = __ldg(reinterpret_cast<const float4 *>(a.nodes + cur));
    const float4 n1 = __ldg(reinterpret_cast<const float4 *>(a.nodes + cur) + 1);
    // the cell's side record, fetched alongside (unused for leaves)
    const float4 c0 = __ldg(reinterpret_cast<const float4 *>(fa.cells + cur));
    const uint4 c1 = __ldg(reinterpret_cast<const uint4 *>(fa.cells + cur) + 1);
    const float nmass = n1.x, nsize = n1.y;
    const int32_t nnext = __float_as_int(n1.z), ninfo = __float_as_int(n1.w);
    const bool active = cur >= resume && cur < myEnd;
    const float dx = (n0.x - vxh) + (n0.z - vxl);
    const float dy = (n0.y - vyh) + (n0.w - vyl);
    const float d2 = dx * dx + dy * dy;
    const bool isLeaf = ninfo >= 0;
    const bool massOk = nmass != 0.0f;
    const uint32_t skip = max((uint32_t)nnext, cur + 1u);
    const bool contains = cur <= myLeaf && myLeaf < skip;
    const bool accept = !isLeaf && nsize < d2 && !contains;
    const bool doForce = active && massOk && (isLeaf ? ((uint32_t)ninfo != v) : accept);
    const bool open = active && massOk && !isLeaf && !accept;
    float fx = 0.f, fy = 0.f;
    if (__any_sync(0xffffffffu, doForce && !(d2 > 0.0f))) {  // coincident points: rare
      if (doForce) {
        rep_term<MODEL, OVERLAP>(dx, dy, d2, mv, nmass, rv + (isLeaf ? nsize : 0.0f), a.num,
                                 a.overlapC, v, isLeaf ? (uint32_t)ninfo : v, fx, fy);
        kx.add(fx);
        ky.add(fy);
      }
    } else if (doForce) {
      rep_term_apart<MODEL, OVERLAP>(dx, dy, d2, mv, nmass, rv + (isLeaf ? nsize : 0.0f),
                                     a.num, a.overlapC, fx, fy);
      kx.add(fx);
      ky.add(fy);
    }
    if (COUNT && doForce) nInter++;
    const bool wantMlp = doForce && !isLeaf;
    const uint32_t ball = __ballot_sync(0xffffffffu, wantMlp);
    if (ball) {
      FarCell c;
      c.qa = c0.x;
      c.qb = c0.y;
      c.tr = c0.z;
      c.h = c0.w;
      c.ox = __uint_as_float(c1.x);
      c.oy = __uint_as_float(c1.y);
      c.s0 = c1.z;
      c.s1 = c1.w;
      // the cell seen from the warp centroid (the same bits in every lane)
      const float wdx = (n0.x - wxh) + (n0.z - wxl);
      const float wdy = (n0.y - wyh) + (n0.w - wyl);
      const float wd2 = wdx * wdx + wdy * wdy;
      const bool seenW = nsize < wd2, closeW = wr2 <= spread2 * wd2;
      uint32_t wball = __ballot_sync(0xffffffffu, wantMlp && grouping && seenW && closeW);
      if (__popc(wball) < 2) wball = 0u;
      const bool inW = (wball >> lane) & 1u;
      const bool inL = wantMlp && !inW;
      const uint32_t lball = ball & ~wball;
      const int nG = wball ? 1 : 0;
      if (nG > 0 && qg == kFarTile) {
        __syncwarp();
        mlp_forward_tile<true>(W, q.gx, MLP_XS, reinterpret_cast<float *>(q.out));
        __syncwarp();
#pragma unroll 4
        for (int r = 0; r < kFarTile; r++) far_apply(q.out[r], q.gF[r][lane], corrx, corry);
        __syncwarp();
        qg = 0;
      }
      // one feature pass: each lane for its own row
      if (inW || inL) {
        const float sdx = inW ? wdx : dx, sdy = inW ? wdy : dy, sd2 = inW ? wd2 : d2;
        const float srv = OVERLAP ? (inW ? wrv : rv) : 0.f;
        float f[MLP_IN], e1x, e1y;
        far_features(sdx, sdy, sd2, c, srv, f, e1x, e1y);
        if (inL) {
          const int slot = ql + __popc(lball & ((1u << lane) - 1u));
          far_put_row(q.lx + slot * MLP_XS, f);
          q.lF[slot] = make_float2(fx, fy);
          mine |= 1ull << slot;
        } else if ((uint32_t)(__ffs(wball) - 1) == lane) {
          far_put_row(q.gx + qg * MLP_XS, f);
        }
      }
      if (nG) q.gF[qg][lane] = inW ? make_float2(fx, fy) : make_float2(0.f, 0.f);
      if (COUNT) {
        if (lane == 0) {
          nGroup += nG;
          nEvent++;
        }
        if (inL) {
          nLane++;
          nWhy[!seenW ? 2 : (!closeW ? 1 : 0)]++;  // few members / spread / test
        }
      }
      qg += nG;
      ql += __popc(lball);
      while (ql >= kFarTile) {
        __syncwarp();
        mlp_forward_tile<true>(W, q.lx, MLP_XS, reinterpret_cast<float *>(q.out));
        __syncwarp();
        for (uint32_t m = (uint32_t)(mine & 0xffffu); m; m &= m - 1u) {
          const int e = __ffs(m) - 1;
          far_apply(q.out[e], q.lF[e], corrx, corry);
        }
        __syncwarp();
        // move the rows past the tile (at most 31) to the front
        for (int e = kFarTile + (int)lane; e < ql; e += 32) {
          const uint4 *src = reinterpret_cast<const uint4 *>(q.lx + e * MLP_XS);
          uint4 *dst = reinterpret_cast<uint4 *>(q.lx + (e - kFarTile) * MLP_XS);
          dst[0] = src[0];
          dst[1] = src[1];
          q.lF[e - kFarTile] = q.lF[e];
        }
        mine >>= kFarTile;
        ql -= kFarTile;
        __syncwarp();
      }
    }
    if (active) resume = open ? cur + 1u : skip;
    nxt = resume < myEnd ? resume : kInf;
    if (COUNT) nVisit++;
    cur = __reduce_min_sync(0xffffffffu, nxt);
  }
  if (qg > 0) {
    __syncwarp();
    mlp_forward_tile<true>(W, q.gx, MLP_XS, reinterpret_cast<float *>(q.out));
    __syncwarp();
    for (int r = 0; r < qg; r++) far_apply(q.out[r], q.gF[r][lane], corrx, corry);
  }
  if (ql > 0) {
    __syncwarp();
    mlp_forward_tile<true>(W, q.lx, MLP_XS, reinterpret_cast<float *>(q.out));
    __syncwarp();
    for (uint32_t m = (uint32_t)(mine & 0xffffu); m; m &= m - 1u) {
      const int e = __ffs(m) - 1;
      far_apply(q.out[e], q.lF[e], corrx, corry);
    }
  }
  if (COUNT) {
    atomicAdd(a.counters, nInter);
    atomicAdd(a.counters + 3, nLane);
    atomicAdd(a.counters + 4, nWhy[0]);
    atomicAdd(a.counters + 5, nWhy[1]);
    atomicAdd(a.counters + 6, nWhy[2]);
    if (lane == 0) {
      atomicAdd(a.counters + 1, nVisit);
      atomicAdd(a.counters + 2, nGroup);
      atomicAdd(a.counters + 7, nEvent);
    }
  }
  if (!act) return;
  const float2 at = a.attF[v];
  force_epilogue(a.epi, v, (double)at.x, (double)at.y, kx.value() + (double)corrx,
                 ky.value() + (double)corry);
}

// ---------------------------------------------------------------------------
// The learned cell-group walk. One warp per target group cut from the tree
// (k_far_groups: a cell of <= 32 points, sibling cells packed), so the 32
// targets of a warp always lie in one cell and its parent bounds them. The
// warp walks the tree once for the whole group with warp-uniform decisions:
//   point        - every target takes the pair term (self excluded);
//   cell         - opened when its preorder range meets the group's, or when
//                  the opening test fails from the group's bounding box
//                  (2h/theta against the distance from the box to the
//                  cell's centre of mass, the nearest any target can be);
//                  otherwise accepted for every target: each takes its own
//                  monopole term, and one MLP row with the cell seen from
//                  the group's centroid corrects them all (p1 F + p2
//                  rot90(F) with each target's own F).
// Because the decisions do not depend on the target, the warp expands the
// tree 32 cells at a time: each round every lane pops one pending node from
// the warp's stack in shared memory, loads it (32 independent loads instead
// of a chain of dependent ones) and classifies it; points go to a point
// list, accepted cells to a cell list, opened cells push their children
// (their slots come from the tree build's child records). Full lists are
// then evaluated by all 32 lanes, each for its own target: 32 points per
// pass, or 16 cells whose MLP rows form one 16-row mma.sync tile. A push
// that would overflow the stack is walked in place by the warp with the
// stackless preorder loop (same decisions, same lists). The order in which
// terms are summed depends only on the group, so the result does not
// depend on which warp drew it. Per-target sums are Kahan-compensated.
// The lists are at most 63 points and 47 cells: a round adds at most 32 of
// each, and a round runs only while fewer than 32 points and 16 cells wait.
// ---------------------------------------------------------------------------

constexpr int kCellRing = 64;     // point and cell list entries per warp (ring)
constexpr int kCellStack = 512;   // pending nodes per warp
constexpr int kCellThreads = 256; // one block of 8 warps shares the staged network
constexpr int kCellBlocksPerSM = 3;

// per warp: the point and cell lists (double-single positions), the MLP
// tile's rows and outputs, the group's targets and the pending nodes
struct __align__(16) CellWarpSmem {
  float4 pPos[kCellRing];  // point: x hi, y hi, x lo, y lo
  float2 pMR[kCellRing];   // point: mass, radius
  uint32_t pV[kCellRing];  // point: vertex
  float4 cPos[kCellRing];  // cell: centre of mass, double-single
  float2 cMN[kCellRing];   // cell: mass, preorder slot (bits)
  __nv_bfloat16 gx[kFarTile * MLP_XS];
  float2 out[kFarTile];
  uint32_t tgt[32];
  uint32_t st[kCellStack];
};
constexpr size_t kCellDyn = (kCellThreads / 32) * sizeof(CellWarpSmem);

struct CellArgs {
  FarArgs f;
  const uint4 *groups;
  const uint4 *kids;
  const uint32_t *nGroups;  // [0] groups written, [1] the walk's task counter
  uint32_t cap;
  uint32_t stackCap;  // stack entries per warp in use (<= kCellStack)
};

__device__ __forceinline__ float warp_minf(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fminf(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}
__device__ __forceinline__ float warp_maxf(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

// One group's walk state: this lane's target and sums, the group's centroid
// and bounding box, and the warp-uniform list cursors.
struct CellTarget {
  uint32_t v;
  bool has;
  float vxh, vxl, vyh, vyl, mv, rv;
};

struct CellGroup {
  float wxh, wxl, wyh, wyl, wrv;  // centroid (double-single) and mean radius
  float bx0, bx1, by0, by1;       // bounding box of the targets (hi parts)
  uint32_t gx, gy;                // the group's preorder range
};

struct CellSums {
  Kahan kx, ky;
  float corrx = 0.f, corry = 0.f;
  uint32_t ph = 0, pn = 0, ch = 0, cn = 0;  // list heads and lengths
  unsigned long long nInter = 0, nRows = 0;  // instrumentation only
};

// Every target takes the pair term of the first k listed points (at most
// 32, summed in a plain FP32 partial that then joins the target's
// Kahan-compensated sum: cascade summation, as in the plain walk).
template <int MODEL, bool OVERLAP, bool COUNT>
__device__ __forceinline__ void cell_eval_points(const WalkArgs &a, CellWarpSmem &q,
                                                 const CellTarget &t, CellSums &s, uint32_t k) {
  __syncwarp();
  float px = 0.f, py = 0.f;
#pragma unroll 1  // a compact loop: the walk is sensitive to instruction-cache misses
  for (uint32_t j = 0; j < k; j++) {
    const uint32_t e = (s.ph + j) & (kCellRing - 1);
    const float4 p = q.pPos[e];
    const float2 mr = q.pMR[e];
    const uint32_t u = q.pV[e];
    const float dx = (p.x - t.vxh) + (p.z - t.vxl);
    const float dy = (p.y - t.vyh) + (p.w - t.vyl);
    const float d2 = dx * dx + dy * dy;
    const bool doForce = t.has && u != t.v;
    float fx = 0.f, fy = 0.f;
    if (__any_sync(0xffffffffu, doForce && !(d2 > 0.0f))) {  // coincident points: rare
      if (doForce)
        rep_term<MODEL, OVERLAP>(dx, dy, d2, t.mv, mr.x, t.rv + mr.y, a.num, a.overlapC, t.v,
                                 u, fx, fy);
    } else if (doForce) {
      rep_term_apart<MODEL, OVERLAP>(dx, dy, d2, t.mv, mr.x, t.rv + mr.y, a.num, a.overlapC,
                                     fx, fy);
    }
    px += fx;
    py += fy;
    if (COUNT && doForce) s.nInter++;
  }
  s.kx.add(px);
  s.ky.add(py);
  s.ph = (s.ph + k) & (kCellRing - 1);
  s.pn -= k;
  __syncwarp();
}

// The first k <= 16 listed cells: lane r < k builds row r (cell r seen from
// the group's centroid), the tile runs on the tensor cores, then every
// target adds each cell's monopole term (a plain partial of the k terms,
// then the Kahan sum) and the row's correction of it.
template <int MODEL, bool OVERLAP, bool COUNT>
__device__ __forceinline__ void cell_eval_cells(const WalkArgs &a, const FarCell *__restrict__ cells,
                                                const MlpSmem &W, CellWarpSmem &q,
                                                const CellTarget &t, const CellGroup &g,
                                                CellSums &s, uint32_t k) {
  const uint32_t lane = threadIdx.x & 31u;
  __syncwarp();
  if (lane < k) {
    const uint32_t e = (s.ch + lane) & (kCellRing - 1);
    const float4 p = q.cPos[e];
    const uint32_t node = __float_as_uint(q.cMN[e].y);
    const float4 c0 = __ldg(reinterpret_cast<const float4 *>(cells + node));
    const uint4 c1 = __ldg(reinterpret_cast<const uint4 *>(cells + node) + 1);
    FarCell c;
    c.qa = c0.x;
    c.qb = c0.y;
    c.tr = c0.z;
    c.h = c0.w;
    c.ox = __uint_as_float(c1.x);
    c.oy = __uint_as_float(c1.y);
    c.s0 = c1.z;
    c.s1 = c1.w;
    const float wdx = (p.x - g.wxh) + (p.z - g.wxl);
    const float wdy = (p.y - g.wyh) + (p.w - g.wyl);
    const float wd2 = wdx * wdx + wdy * wdy;
    float f[MLP_IN], e1x, e1y;
    far_features(wdx, wdy, wd2, c, OVERLAP ? g.wrv : 0.f, f, e1x, e1y);
    far_put_row(q.gx + lane * MLP_XS, f);
  }
  __syncwarp();
  mlp_forward_tile<true>(W, q.gx, MLP_XS, reinterpret_cast<float *>(q.out));
  __syncwarp();
  float px = 0.f, py = 0.f;
#pragma unroll 1  // a compact loop: the walk is sensitive to instruction-cache misses
  for (uint32_t r = 0; r < k; r++) {
    const uint32_t e = (s.ch + r) & (kCellRing - 1);
    const float4 p = q.cPos[e];
    const float m = q.cMN[e].x;
    const float dx = (p.x - t.vxh) + (p.z - t.vxl);
    const float dy = (p.y - t.vyh) + (p.w - t.vyl);
    const float d2 = dx * dx + dy * dy;
    float fx = 0.f, fy = 0.f;
    if (__any_sync(0xffffffffu, t.has && !(d2 > 0.0f))) {
      if (t.has)
        rep_term<MODEL, OVERLAP>(dx, dy, d2, t.mv, m, t.rv, a.num, a.overlapC, t.v, t.v, fx, fy);
    } else if (t.has) {
      rep_term_apart<MODEL, OVERLAP>(dx, dy, d2, t.mv, m, t.rv, a.num, a.overlapC, fx, fy);
    }
    px += fx;
    py += fy;
    if (t.has) {
      far_apply(q.out[r], make_float2(fx, fy), s.corrx, s.corry);
      if (COUNT) s.nInter++;
    }
  }
  s.kx.add(px);
  s.ky.add(py);
  if (COUNT) s.nRows += k;
  s.ch = (s.ch + k) & (kCellRing - 1);
  s.cn -= k;
  __syncwarp();
}

// Classification of node `cur` (record n0, n1) for the group: 0 nothing
// (empty), 1 point, 2 accepted cell, 3 opened cell.
__device__ __forceinline__ int cell_classify(const CellGroup &g, uint32_t cur, float4 n0,
                                             float4 n1) {
  const float nmass = n1.x, nsize = n1.y;
  const int32_t nnext = __float_as_int(n1.z), ninfo = __float_as_int(n1.w);
  if (nmass == 0.0f) return 0;  // empty: skipped as the reference does
  if (ninfo >= 0) return 1;
  const uint32_t skip = max((uint32_t)nnext, cur + 1u);
  if (cur < g.gy && skip > g.gx) return 3;  // holds targets of the group
  const float ex = fmaxf(fmaxf(g.bx0 - n0.x, n0.x - g.bx1), 0.0f);
  const float ey = fmaxf(fmaxf(g.by0 - n0.y, n0.y - g.by1), 0.0f);
  return nsize < ex * ex + ey * ey ? 2 : 3;
}

template <int MODEL, bool OVERLAP, bool COUNT>
__global__ __launch_bounds__(kCellThreads, kCellBlocksPerSM) void k_walk_f32_cells(CellArgs ca) {
  __shared__ MlpSmem W;
  extern __shared__ __align__(16) unsigned char cellDyn[];
  CellWarpSmem *Q = reinterpret_cast<CellWarpSmem *>(cellDyn);  // one per warp
  mlp_stage(W, ca.f.mlp);
  const WalkArgs &a = ca.f.w;
  const FarCell *__restrict__ cells = ca.f.cells;
  const uint4 *__restrict__ kids = ca.kids;
  CellWarpSmem &q = Q[threadIdx.x >> 5];
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t below = (1u << lane) - 1u;
  for (int e = lane; e < kFarTile * MLP_XS / 8; e += 32)
    reinterpret_cast<uint4 *>(q.gx)[e] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  const uint32_t nGroups = min(ca.nGroups[0], ca.cap);
  uint32_t *queue = const_cast<uint32_t *>(ca.nGroups) + 1;
  unsigned long long nInter = 0, nVisit = 0, nRows = 0, nGrp = 0, nSerial = 0;
  for (;;) {
    uint32_t gi = 0;
    if (lane == 0) gi = atomicAdd(queue, 1u);
    gi = __shfl_sync(0xffffffffu, gi, 0);
    if (gi >= nGroups) break;
    const uint4 G = ca.groups[gi];
    // the group's targets: the leaves of its preorder range, one per lane
    uint32_t found = 0;
    for (uint32_t b = G.x; b < G.y && found < 32u; b += 32u) {
      const uint32_t j = b + lane;
      const int32_t info = j < G.y ? __ldg(reinterpret_cast<const int4 *>(a.nodes + j) + 1).w : -1;
      const uint32_t ball = __ballot_sync(0xffffffffu, info >= 0);
      const uint32_t r = found + __popc(ball & below);
      if (info >= 0 && r < 32u) q.tgt[r] = (uint32_t)info;
      found += __popc(ball);
    }
    __syncwarp();
    const uint32_t nT = min(found, 32u);
    CellTarget t;
    t.has = lane < nT;
    t.v = t.has ? q.tgt[lane] : 0u;
    __syncwarp();
    if (nT == 0) continue;
    const uint32_t v0 = __shfl_sync(0xffffffffu, t.v, 0);
    const uint32_t gr = a.gid ? a.gid[v0] : 0u;
    if (a.active && a.active[gr] == 0u) continue;
    const uint32_t root = a.graphBase[gr];
    const uint32_t end = min(root + a.rootT[gr], a.maxNodes);
    t.vxh = t.vxl = t.vyh = t.vyl = t.mv = t.rv = 0.f;
    double2 pv = make_double2(0.0, 0.0);
    if (t.has) {
      pv = a.pos[t.v];
      ds_split(pv.x, t.vxh, t.vxl);
      ds_split(pv.y, t.vyh, t.vyl);
      t.mv = a.massF[t.v];
      if (OVERLAP) t.rv = a.radiusF[t.v];
    }
    CellGroup g;
    float wr2;
    group_centroid<32, OVERLAP>(t.has, pv, t.vxh, t.vxl, t.vyh, t.vyl, t.rv, g.wxh, g.wxl,
                                g.wyh, g.wyl, wr2, g.wrv);
    g.bx0 = warp_minf(t.has ? t.vxh : INFINITY);
    g.bx1 = warp_maxf(t.has ? t.vxh : -INFINITY);
    g.by0 = warp_minf(t.has ? t.vyh : INFINITY);
    g.by1 = warp_maxf(t.has ? t.vyh : -INFINITY);
    g.gx = G.x;
    g.gy = G.y;
    CellSums s;
    const unsigned long long visit0 = nVisit;
    if (COUNT) nGrp++;
    // pending nodes (stack), the in-place walk of a subtree that did not
    // fit the stack [serCur, serEnd), and the lanes whose subtrees wait for
    // it (each holds its range in sLo, sHi); all warp-uniform but sLo/sHi
    uint32_t top = 0, serCur = 0, serEnd = 0, pendS = 0, sLo = 0, sHi = 0;
    if (root < end) {
      if (lane == 0) q.st[0] = root;
      top = 1;
    }
    __syncwarp();
    // Each pass either evaluates a full list (or, once nothing is left to
    // expand, what remains) or expands more of the tree.
    for (;;) {
      const bool more = serCur < serEnd || pendS != 0u || top > 0u;
      if (s.pn >= 32u || (!more && s.pn > 0u)) {
        cell_eval_points<MODEL, OVERLAP, COUNT>(a, q, t, s, min(s.pn, 32u));
        continue;
      }
      if (s.cn >= (uint32_t)kFarTile || (!more && s.cn > 0u)) {
        cell_eval_cells<MODEL, OVERLAP, COUNT>(a, cells, W, q, t, g, s,
                                               min(s.cn, (uint32_t)kFarTile));
        continue;
      }
      if (!more) break;
      if (serCur < serEnd) {
        // the stackless preorder walk, one node at a time, until a list fills
        while (serCur < serEnd && s.pn < 32u && s.cn < (uint32_t)kFarTile) {
          const uint32_t cur = serCur;
          const float4 n0 = __ldg(reinterpret_cast<const float4 *>(a.nodes + cur));
          const float4 n1 = __ldg(reinterpret_cast<const float4 *>(a.nodes + cur) + 1);
          const uint32_t skip = min(max((uint32_t)__float_as_int(n1.z), cur + 1u), serEnd);
          if (COUNT) nVisit++;
          const int kind = cell_classify(g, cur, n0, n1);
          if (kind == 1 && lane == 0) {
            const uint32_t e = (s.ph + s.pn) & (kCellRing - 1);
            q.pPos[e] = n0;
            q.pMR[e] = make_float2(n1.x, n1.y);
            q.pV[e] = (uint32_t)__float_as_int(n1.w);
          }
          if (kind == 2 && lane == 0) {
            const uint32_t e = (s.ch + s.cn) & (kCellRing - 1);
            q.cPos[e] = n0;
            q.cMN[e] = make_float2(n1.x, __uint_as_float(cur));
          }
          s.pn += kind == 1 ? 1u : 0u;
          s.cn += kind == 2 ? 1u : 0u;
          serCur = kind == 3 ? cur + 1u : skip;
        }
        continue;
      }
      if (pendS) {
        const int l = __ffs(pendS) - 1;
        pendS &= pendS - 1u;
        serCur = __shfl_sync(0xffffffffu, sLo, l);
        serEnd = __shfl_sync(0xffffffffu, sHi, l);
        if (COUNT) nSerial++;
        continue;
      }
      // one expansion round: up to 32 pending nodes, one per lane
      const uint32_t n = min(top, 32u);
      const bool mine = lane < n;
      const uint32_t cur = mine ? q.st[top - n + lane] : 0u;
      top -= n;
      __syncwarp();  // popped before the pushes below reuse the slots
      float4 n0 = make_float4(0.f, 0.f, 0.f, 0.f), n1 = n0;
      uint4 kd = make_uint4(GVIZ_NONE, GVIZ_NONE, GVIZ_NONE, GVIZ_NONE);
      if (mine) {
        n0 = __ldg(reinterpret_cast<const float4 *>(a.nodes + cur));
        n1 = __ldg(reinterpret_cast<const float4 *>(a.nodes + cur) + 1);
        kd = __ldg(kids + cur);  // read for every node; used only when it is opened
      }
      if (COUNT) nVisit += n;
      const int kind = mine ? cell_classify(g, cur, n0, n1) : 0;
      // children inside (cur, end) only: a child record never sends the
      // walk outside the graph's subtree
      uint32_t nk = 0;
      if (kind == 3) {
        if (kd.y == GVIZ_KIDS_RUN) {
          nk = (kd.x > cur && kd.x < end) ? min(kd.z, end - kd.x) : 0u;
          nk = min(nk, (uint32_t)kCellStack + 1u);  // a longer run never fits
          kd.w = 0u;
        } else {
          kd.x = (kd.x > cur && kd.x < end) ? kd.x : GVIZ_NONE;
          kd.y = (kd.y > cur && kd.y < end) ? kd.y : GVIZ_NONE;
          kd.z = (kd.z > cur && kd.z < end) ? kd.z : GVIZ_NONE;
          kd.w = (kd.w > cur && kd.w < end) ? kd.w : GVIZ_NONE;
          nk = (uint32_t)(kd.x != GVIZ_NONE) + (uint32_t)(kd.y != GVIZ_NONE) +
               (uint32_t)(kd.z != GVIZ_NONE) + (uint32_t)(kd.w != GVIZ_NONE);
        }
      }
      // points and accepted cells join their lists in lane order
      const uint32_t bP = __ballot_sync(0xffffffffu, kind == 1);
      if (kind == 1) {
        const uint32_t e = (s.ph + s.pn + __popc(bP & below)) & (kCellRing - 1);
        q.pPos[e] = n0;
        q.pMR[e] = make_float2(n1.x, n1.y);
        q.pV[e] = (uint32_t)__float_as_int(n1.w);
      }
      s.pn += __popc(bP);
      const uint32_t bC = __ballot_sync(0xffffffffu, kind == 2);
      if (kind == 2) {
        const uint32_t e = (s.ch + s.cn + __popc(bC & below)) & (kCellRing - 1);
        q.cPos[e] = n0;
        q.cMN[e] = make_float2(n1.x, __uint_as_float(cur));
      }
      s.cn += __popc(bC);
      // opened cells push their children (lane order) while they fit; the
      // rest wait for the in-place walk
      uint32_t incl = nk;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      const bool fits = top + incl <= ca.stackCap;
      if (kind == 3 && fits) {
        const uint32_t base = top + incl - nk;
        if (kd.y == GVIZ_KIDS_RUN) {
          for (uint32_t i = 0; i < nk; i++) q.st[base + i] = kd.x + i;
        } else {
          uint32_t w = base;
          if (kd.x != GVIZ_NONE) q.st[w++] = kd.x;
          if (kd.y != GVIZ_NONE) q.st[w++] = kd.y;
          if (kd.z != GVIZ_NONE) q.st[w++] = kd.z;
          if (kd.w != GVIZ_NONE) q.st[w++] = kd.w;
        }
      }
      top += __reduce_max_sync(0xffffffffu, fits ? incl : 0u);
      pendS = __ballot_sync(0xffffffffu, kind == 3 && !fits);
      if (kind == 3 && !fits) {
        sLo = cur + 1u;
        sHi = min(max((uint32_t)__float_as_int(n1.z), cur + 1u), end);
      }
      __syncwarp();
    }
    if (COUNT) {
      nInter += s.nInter;
      if (lane == 0) {
        nRows += s.nRows;
        const unsigned long long len = nVisit - visit0;
        atomicMax(a.counters + 4, len);  // the longest group walk
        atomicAdd(a.counters + 6, (unsigned long long)nT);
      }
    }
    if (t.has) {
      const float2 at = a.attF[t.v];
      force_epilogue(a.epi, t.v, (double)at.x, (double)at.y, s.kx.value() + (double)s.corrx,
                     s.ky.value() + (double)s.corry);
    }
  }
  if (COUNT) {
    atomicAdd(a.counters, nInter);
    if (lane == 0) {
      atomicAdd(a.counters + 1, nVisit);
      atomicAdd(a.counters + 2, nRows);
      atomicAdd(a.counters + 5, nSerial);
      atomicAdd(a.counters + 7, nGrp);
    }
  }
}
// ---------------------------------------------------------------------------
// Hub targets of the learned walk. LinLog's pair force scales with the
// target's mass, so the heaviest targets carry most of the force and their
// errors dominate the force-weighted RMS error. They are walked again with
// the plain monopole method at a tighter opening threshold (farHubTheta) and
// their learned results replaced. One warp walks one hub (hubs are drawn
// from a counter) through a first-in first-out ring of preorder ranges
// [lo, hi) of consecutive sibling subtrees in shared memory: a lane takes
// kHubTake entries per round, loads their first nodes together, tests them
// (leaf: pair term; cell: accepted, or opened) and yields at most two
// entries for each, the opened cell's children [lo + 1, next) and the
// remaining siblings [next, hi), appended in lane order after a warp scan.
// An entry that finds the ring full is walked to its end by its lane. A
// hub's sum depends only on the hub, so it is deterministic. The walk is
// bound by the latency of the node loads along the ring, not by bandwidth.
// ---------------------------------------------------------------------------
constexpr int kHubThreads = 128;
constexpr uint32_t kHubRing = 1024;  // ring entries per warp
constexpr int kHubTake = 2;          // entries a lane takes per round

struct FarHubArgs {
  WalkArgs w;
  const uint32_t *hubs;  // vertex ids
  uint32_t *counter;     // hubs drawn so far (reset before every launch)
  double2 *out;          // per hub: its plain repulsion
  uint32_t nHubs;
  float sizeScale;       // (theta / farHubTheta)^2: node sizes hold (2h/theta)^2
};

struct HubTarget {
  uint32_t v;
  float xh, xl, yh, yl, m, r;
};

struct HubNode {
  float4 n0, n1;  // {x hi, y hi, x lo, y lo}, {mass, size, next, info}
};

__device__ __forceinline__ HubNode hub_load(const FarHubArgs &a, uint32_t cur) {
  HubNode n;
  n.n0 = __ldg(reinterpret_cast<const float4 *>(a.w.nodes + cur));
  n.n1 = __ldg(reinterpret_cast<const float4 *>(a.w.nodes + cur) + 1);
  return n;
}

// Tests node `cur` for the hub: adds its term when it is a leaf other than
// the hub or an accepted cell; returns true when the cell is opened. `next`
// is the node after its subtree.
template <int MODEL, bool OVERLAP>
__device__ __forceinline__ bool hub_visit(const FarHubArgs &a, const HubTarget &t, uint32_t cur,
                                          const HubNode &n, Kahan &kx, Kahan &ky,
                                          uint32_t &next) {
  const float nmass = n.n1.x, nsize = n.n1.y;
  const int32_t nnext = __float_as_int(n.n1.z), ninfo = __float_as_int(n.n1.w);
  next = max((uint32_t)nnext, cur + 1u);
  if (nmass == 0.0f) return false;
  const float dx = (n.n0.x - t.xh) + (n.n0.z - t.xl);
  const float dy = (n.n0.y - t.yh) + (n.n0.w - t.yl);
  const float d2 = dx * dx + dy * dy;
  const bool isLeaf = ninfo >= 0;
  if (isLeaf ? (uint32_t)ninfo != t.v : nsize * a.sizeScale < d2) {
    float fx, fy;
    rep_term<MODEL, OVERLAP>(dx, dy, d2, t.m, nmass, t.r + (isLeaf ? nsize : 0.0f), a.w.num,
                             a.w.overlapC, t.v, isLeaf ? (uint32_t)ninfo : t.v, fx, fy);
    kx.add(fx);
    ky.add(fy);
    return false;
  }
  return !isLeaf;
}

// The stackless walk of [lo, hi) by one lane (every step moves forward).
template <int MODEL, bool OVERLAP>
__device__ __forceinline__ void hub_walk_range(const FarHubArgs &a, const HubTarget &t,
                                               uint32_t lo, uint32_t hi, Kahan &kx, Kahan &ky) {
  uint32_t cur = lo;
  while (cur < hi) {
    uint32_t next;
    cur = hub_visit<MODEL, OVERLAP>(a, t, cur, hub_load(a, cur), kx, ky, next) ? cur + 1u : next;
  }
}

template <int MODEL, bool OVERLAP>
__global__ __launch_bounds__(kHubThreads) void k_walk_f32_hubs(FarHubArgs a) {
  __shared__ uint2 ring[kHubThreads / 32][kHubRing];
  const uint32_t lane = threadIdx.x & 31u;
  uint2 *q = ring[threadIdx.x >> 5];
  for (;;) {
    uint32_t i = 0;
    if (lane == 0u) i = atomicAdd(a.counter, 1u);
    i = __shfl_sync(0xffffffffu, i, 0);
    if (i >= a.nHubs) return;
    HubTarget t;
    t.v = a.hubs[i];
    const uint32_t g = a.w.gid ? a.w.gid[t.v] : 0u;
    if (a.w.active && a.w.active[g] == 0u) continue;  // the whole warp
    const uint32_t base = a.w.graphBase[g];
    const uint32_t end = min(base + a.w.rootT[g], a.w.maxNodes);
    const double2 p = a.w.pos[t.v];
    ds_split(p.x, t.xh, t.xl);
    ds_split(p.y, t.yh, t.yl);
    t.m = a.w.massF[t.v];
    t.r = OVERLAP ? a.w.radiusF[t.v] : 0.0f;
    Kahan kx, ky;
    // head, tail: entries taken and appended so far (warp-uniform)
    uint32_t head = 0, tail = base < end ? 1u : 0u;
    if (lane == 0u) q[0] = make_uint2(base, end);
    __syncwarp();
    while (head < tail) {
      const uint32_t take = min(tail - head, 32u * kHubTake);
      uint2 r[kHubTake];
      HubNode n[kHubTake];
#pragma unroll
      for (int u = 0; u < kHubTake; u++) {
        const uint32_t k = lane + 32u * u;
        r[u] = k < take ? q[(head + k) % kHubRing] : make_uint2(0u, 0u);
        if (k < take) n[u] = hub_load(a, r[u].x);
      }
      // each taken entry yields its children and / or its remaining siblings
      uint2 e[2 * kHubTake];
      uint32_t c = 0;
#pragma unroll
      for (int u = 0; u < kHubTake; u++) {
        e[2 * u] = e[2 * u + 1] = make_uint2(0u, 0u);
        if (lane + 32u * u < take) {
          uint32_t next;
          const bool open = hub_visit<MODEL, OVERLAP>(a, t, r[u].x, n[u], kx, ky, next);
          const uint32_t childEnd = min(next, r[u].y);  // entries stay inside [base, end)
          if (open && r[u].x + 1u < childEnd) e[2 * u] = make_uint2(r[u].x + 1u, childEnd);
          if (next < r[u].y) e[2 * u + 1] = make_uint2(next, r[u].y);
        }
        c += (uint32_t)(e[2 * u].x < e[2 * u].y) + (uint32_t)(e[2 * u + 1].x < e[2 * u + 1].y);
      }
      __syncwarp();  // the slots just read are free from here on
      head += take;
      uint32_t incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
      const uint32_t room = kHubRing - (tail - head);
      uint32_t slot = incl - c;
#pragma unroll
      for (int k = 0; k < 2 * kHubTake; k++) {
        if (!(e[k].x < e[k].y)) continue;  // an empty range is no entry
        if (slot < room) q[(tail + slot) % kHubRing] = e[k];
        else hub_walk_range<MODEL, OVERLAP>(a, t, e[k].x, e[k].y, kx, ky);
        slot++;
      }
      tail += min(total, room);
      __syncwarp();
    }
    double sx = kx.value(), sy = ky.value();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sx += __shfl_xor_sync(0xffffffffu, sx, o);
      sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    if (lane == 0u) a.out[i] = make_double2(sx, sy);
  }
}

// The hubs' force epilogues with their plain repulsion, after the learned
// walk wrote theirs.
__global__ __launch_bounds__(256) void k_far_hub_epilogue(FarHubArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nHubs) return;
  const uint32_t v = a.hubs[i];
  const uint32_t g = a.w.gid ? a.w.gid[v] : 0u;
  if (a.w.active && a.w.active[g] == 0u) return;
  const float2 at = a.w.attF[v];
  const double2 r = a.out[i];
  force_epilogue(a.w.epi, v, (double)at.x, (double)at.y, r.x, r.y);
}

struct ExactArgs {
  const double2 *pos;
  const float *massF, *radiusF;
  const uint32_t *gid, *active;
  const uint64_t *graphOff;
  const float2 *attF;
  EpiArgs epi;
  float num, overlapC;
  uint32_t V;
  double2 *partial;  // [splits][V] per-split sums (splits > 1)
  uint32_t splits;
};

// Exact all-pairs repulsion (src/embedders/gvizForceEmbedder.c:104-115) as
// a tiled N-body: a block holds kExactThreads * kExactTpt targets, each
// thread kExactTpt of them (kExactThreads apart), and the sources stream
// through shared memory in tiles of kExactTile; every source read from
// shared memory serves kExactTpt targets. Per target the terms of each run
// of kExactChunk sources are added in plain FP32 and that partial joins a
// Kahan-compensated running sum (cascade summation: the rounding of a
// V-term sum stays at a chunk's). The pair term runs straight-line; a chunk
// whose sum meets the target itself or a duplicate point (d2 == 0) is summed
// again on the guarded path, which skips the self pair and applies the
// coincident direction. Tiles that straddle a graph boundary of a forest,
// and every tile with overlap prevention, take the guarded path.
// The sources are split into gridDim.y consecutive ranges of whole tiles
// (so that small layouts still fill the GPU); with more than one range each
// block writes its per-target partial sums and k_exact_combine adds them in
// range order.
template <int MODEL, bool OVERLAP>
__global__ __launch_bounds__(kExactThreads) void k_exact_f32(ExactArgs a) {
  __shared__ float4 sp[kExactTile];
  __shared__ float2 sm[kExactTile];
  __shared__ float sw[kExactTile];  // the source's share of the optimistic term's numerator
  __shared__ uint32_t sRange[2];
  uint32_t v[kExactTpt], gb[kExactTpt], ge[kExactTpt];
  bool act[kExactTpt];
  float vxh[kExactTpt], vxl[kExactTpt], vyh[kExactTpt], vyl[kExactTpt], mv[kExactTpt],
      rv[kExactTpt];
  Kahan kx[kExactTpt], ky[kExactTpt];
  if (threadIdx.x == 0) {
    sRange[0] = kInf;
    sRange[1] = 0;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kExactTpt; k++) {
    v[k] = blockIdx.x * (kExactThreads * kExactTpt) + k * kExactThreads + threadIdx.x;
    const bool valid = v[k] < a.V;
    const uint32_t g = (valid && a.gid) ? a.gid[v[k]] : 0u;
    act[k] = valid && (a.active == nullptr || a.active[g] != 0u);
    gb[k] = ge[k] = 0;
    // an idle slot sits at NaN: its terms are never used and never vote
    vxh[k] = vxl[k] = vyh[k] = vyl[k] = __int_as_float(0x7fc00000);
    mv[k] = rv[k] = 0.f;
    if (act[k]) {
      gb[k] = (uint32_t)a.graphOff[g];
      ge[k] = (uint32_t)a.graphOff[g + 1];
      atomicMin(&sRange[0], gb[k]);
      atomicMax(&sRange[1], ge[k]);
      const double2 p = a.pos[v[k]];
      ds_split(p.x, vxh[k], vxl[k]);
      ds_split(p.y, vyh[k], vyl[k]);
      mv[k] = a.massF[v[k]];
      if (OVERLAP) rv[k] = a.radiusF[v[k]];
    }
  }
  __syncthreads();
  const uint32_t lo = sRange[0], hi = sRange[1];
  // this block's source range: whole tiles, split blockIdx.y of gridDim.y
  const uint32_t nTile = hi > lo ? (hi - lo + kExactTile - 1) / kExactTile : 0u;
  const uint32_t per = (nTile + gridDim.y - 1) / gridDim.y;
  const uint32_t s0 = lo + min(blockIdx.y * per, nTile) * kExactTile;
  const uint32_t s1 = min(hi, lo + min((blockIdx.y + 1) * per, nTile) * kExactTile);
  for (uint32_t t0 = s0; t0 < s1; t0 += kExactTile) {
    __syncthreads();
    const uint32_t j = t0 + threadIdx.x;
    if (threadIdx.x < kExactTile && j < hi) {
      const double2 q = a.pos[j];
      float4 f;
      ds_split(q.x, f.x, f.z);
      ds_split(q.y, f.y, f.w);
      sp[threadIdx.x] = f;
      const float m = a.massF[j];
      sm[threadIdx.x] = make_float2(m, OVERLAP ? a.radiusF[j] : 0.f);
      sw[threadIdx.x] = MODEL == GVIZ_CUDA_MODEL_FR ? a.num * truncf(m) : m;
    }
    __syncthreads();
    const uint32_t cnt = min((uint32_t)kExactTile, hi - t0);
    bool inside = true;  // the whole tile lies in every target's graph
#pragma unroll
    for (int k = 0; k < kExactTpt; k++)
      inside = inside && (!act[k] || (gb[k] <= t0 && t0 + cnt <= ge[k]));
    const bool fastTile = __all_sync(0xffffffffu, inside);
    for (uint32_t c0 = 0; c0 < cnt; c0 += kExactChunk) {
      const uint32_t c1 = min(c0 + (uint32_t)kExactChunk, cnt);
      float px[kExactTpt], py[kExactTpt];
#pragma unroll
      for (int k = 0; k < kExactTpt; k++) px[k] = py[k] = 0.f;
      bool redo = true;
      if (!OVERLAP && fastTile) {
        // Optimistic: without overlap the term is numer / d2 along (dx, dy),
        // with the source's share of the numerator taken once per source
        // (FR: k^2 times the truncated mass, src/embedders/gvizForceModel.c:20;
        // LinLog: its mass), one approximate reciprocal per pair, and the
        // term fused into the chunk's partial. The reciprocal is the PTX
        // instruction rcp.approx.ftz.f32 (one MUFU op, no range handling):
        // the self pair, a coincident point (d2 == 0) or a d2 below the
        // normal range (flushed to zero) gives an infinite term, so the
        // chunk's partial is not finite and the chunk is summed again on
        // the guarded path below.
#pragma unroll 4
        for (uint32_t q = c0; q < c1; q++) {
          const float4 f = sp[q];
          const float w = sw[q];
#pragma unroll
          for (int k = 0; k < kExactTpt; k++) {
            const float dx = (f.x - vxh[k]) + (f.z - vxl[k]);
            const float dy = (f.y - vyh[k]) + (f.w - vyl[k]);
            const float sc = w * rcp_approx_ftz(dx * dx + dy * dy);
            px[k] = fmaf(-sc, dx, px[k]);
            py[k] = fmaf(-sc, dy, py[k]);
          }
        }
        // LinLog's target mass is common to the chunk's terms: one multiply
        // per chunk instead of one per pair
        if (MODEL != GVIZ_CUDA_MODEL_FR) {
#pragma unroll
          for (int k = 0; k < kExactTpt; k++) {
            px[k] *= mv[k];
            py[k] *= mv[k];
          }
        }
        bool bad = false;
#pragma unroll
        for (int k = 0; k < kExactTpt; k++)
          bad = bad || (act[k] && !(isfinite(px[k]) && isfinite(py[k])));
        redo = __any_sync(0xffffffffu, bad);
        if (redo) {
#pragma unroll
          for (int k = 0; k < kExactTpt; k++) px[k] = py[k] = 0.f;
        }
      }
      if (redo) {
        // guarded: the graph ranges of a forest, the self pair skipped, a
        // coincident point through the deterministic direction; with
        // overlap the term of include/core/gvizVec.h:404-428 / 552-578
        for (uint32_t q = c0; q < c1; q++) {
          const float4 f = sp[q];
          const float2 m = sm[q];
          const uint32_t jj = t0 + q;
          float dx[kExactTpt], dy[kExactTpt], d2[kExactTpt];
          bool zero = false;
#pragma unroll
          for (int k = 0; k < kExactTpt; k++) {
            dx[k] = (f.x - vxh[k]) + (f.z - vxl[k]);
            dy[k] = (f.y - vyh[k]) + (f.w - vyl[k]);
            d2[k] = dx[k] * dx[k] + dy[k] * dy[k];
            zero = zero || (act[k] && d2[k] == 0.0f);
          }
          if (fastTile && !__any_sync(0xffffffffu, zero)) {
#pragma unroll
            for (int k = 0; k < kExactTpt; k++) {
              float fx, fy;
              rep_term_apart<MODEL, OVERLAP>(dx[k], dy[k], d2[k], mv[k], m.x, rv[k] + m.y,
                                             a.num, a.overlapC, fx, fy);
              px[k] += fx;
              py[k] += fy;
            }
          } else {
#pragma unroll
            for (int k = 0; k < kExactTpt; k++) {
              if (!act[k] || jj == v[k] || jj < gb[k] || jj >= ge[k]) continue;
              float fx, fy;
              rep_term<MODEL, OVERLAP>(dx[k], dy[k], d2[k], mv[k], m.x, rv[k] + m.y, a.num,
                                       a.overlapC, v[k], jj, fx, fy);
              px[k] += fx;
              py[k] += fy;
            }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < kExactTpt; k++) {
        kx[k].add(px[k]);
        ky[k].add(py[k]);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kExactTpt; k++) {
    if (!act[k]) continue;
    if (gridDim.y > 1) {
      a.partial[(size_t)blockIdx.y * a.V + v[k]] = make_double2(kx[k].value(), ky[k].value());
      continue;
    }
    const float2 at = a.attF[v[k]];
    force_epilogue(a.epi, v[k], (double)at.x, (double)at.y, kx[k].value(), ky[k].value());
  }
}

// The split sums of each target added in range order, then its epilogue.
__global__ __launch_bounds__(256) void k_exact_combine(ExactArgs a) {
  const uint32_t v = blockIdx.x * 256 + threadIdx.x;
  if (v >= a.V) return;
  const uint32_t g = a.gid ? a.gid[v] : 0u;
  if (a.active && a.active[g] == 0u) return;
  double sx = 0.0, sy = 0.0;
  for (uint32_t s = 0; s < a.splits; s++) {
    const double2 p = a.partial[(size_t)s * a.V + v];
    sx += p.x;
    sy += p.y;
  }
  const float2 at = a.attF[v];
  force_epilogue(a.epi, v, (double)at.x, (double)at.y, sx, sy);
}

inline uint32_t blocks(size_t n, int t) { return (uint32_t)((n + t - 1) / t); }

}  // namespace

void enqueue_attraction_f32(gvizCudaForce *h) {
  AttrArgs a;
  a.rowOff = h->d_rowOff;
  a.cols = h->d_cols;
  a.gid = h->d_gid;
  a.active = h->d_active;
  a.pos = h->d_pos;
  a.out = h->d_attF;
  a.invK = (float)(1.0 / h->params.edgeLength);
  const bool fr = h->model == GVIZ_CUDA_MODEL_FR;
  if (h->nAttrLight) {
    a.list = h->d_attrLight;
    a.n = h->nAttrLight;
    const uint32_t g = blocks(a.n, kAttrThreads);
    if (fr) k_attr_f32_light<GVIZ_CUDA_MODEL_FR><<<g, kAttrThreads, 0, h->stream>>>(a);
    else k_attr_f32_light<GVIZ_CUDA_MODEL_LINLOG><<<g, kAttrThreads, 0, h->stream>>>(a);
  }
  if (h->nAttrHeavy) {
    a.list = h->d_attrHeavy;
    a.n = h->nAttrHeavy;
    const uint32_t g = blocks((size_t)a.n * 32, kAttrThreads);
    if (fr) k_attr_f32_heavy<GVIZ_CUDA_MODEL_FR><<<g, kAttrThreads, 0, h->stream>>>(a);
    else k_attr_f32_heavy<GVIZ_CUDA_MODEL_LINLOG><<<g, kAttrThreads, 0, h->stream>>>(a);
  }
  if (h->nHubs) {
    HubArgs b;
    b.rowOff = h->d_rowOff;
    b.cols = h->d_cols;
    b.gid = h->d_gid;
    b.active = h->d_active;
    b.chunkV = h->d_hubChunkV;
    b.chunkE0 = h->d_hubChunkE0;
    b.chunkE1 = h->d_hubChunkE1;
    b.hubV = h->d_hubV;
    b.hubFirst = h->d_hubFirst;
    b.pos = h->d_pos;
    b.partial = h->d_hubPartial;
    b.out = h->d_attF;
    b.invK = a.invK;
    b.nChunks = h->nHubChunks;
    b.nHubs = h->nHubs;
    const uint32_t g = blocks((size_t)b.nChunks * 32, kAttrThreads);
    if (fr) k_attr_f32_hub_chunks<GVIZ_CUDA_MODEL_FR><<<g, kAttrThreads, 0, h->stream>>>(b);
    else k_attr_f32_hub_chunks<GVIZ_CUDA_MODEL_LINLOG><<<g, kAttrThreads, 0, h->stream>>>(b);
    k_attr_hub_sum<<<blocks(b.nHubs, kAttrThreads), kAttrThreads, 0, h->stream>>>(b);
  }
  prof_mark(h, "attraction_f32");
}

// the plain walk's stack entries per warp on this handle: the caller's cap
// (gvizCudaForceSetWalkStackCap), else the autotuner's pick, else all 512
uint32_t plain_cap(const gvizCudaForce *h) {
  const uint32_t c = h->walkStackCap ? h->walkStackCap : h->walkTunedCap;
  return (c >= 32 && c <= (uint32_t)kPlainStack) ? c : (uint32_t)kPlainStack;
}

// dynamic shared memory of the plain walk: one warp region per warp
static size_t plain_smem(uint32_t threads, uint32_t cap) {
  return (size_t)(threads / 32) * plain_warp_bytes(cap);
}

template <int MODEL, bool OVERLAP, bool COUNT>
static void launch_walk(gvizCudaForce *h, const WalkArgs &a) {
  const uint32_t threads = h->walkThreads ? h->walkThreads : kWalkThreads;
  const uint32_t warps = h->nWalkTasks;
  if (warps == 0) return;
  if (h->walkPersistent && h->walkResident) {
    cudaMemsetAsync(a.queue, 0, sizeof(uint32_t), h->stream);
    const uint32_t need = blocks((size_t)warps * 32, threads);
    const uint32_t grid = need < h->walkResident ? need : h->walkResident;
    k_walk_f32_queue<MODEL, OVERLAP, COUNT><<<grid, threads, plain_smem(threads, a.stackCap),
                                              h->stream>>>(a);
    return;
  }
  k_walk_f32<MODEL, OVERLAP, COUNT><<<blocks((size_t)warps * 32, threads), threads,
                                      plain_smem(threads, a.stackCap), h->stream>>>(a);
}

template <int MODEL, bool OVERLAP>
static void launch_far(gvizCudaForce *h, const FarArgs &fa, bool count) {
  const uint32_t grid = blocks(((h->V + 31) / 32) * 32, kFarThreads);
  if (count) k_walk_f32_far<MODEL, OVERLAP, true><<<grid, kFarThreads, 0, h->stream>>>(fa);
  else k_walk_f32_far<MODEL, OVERLAP, false><<<grid, kFarThreads, 0, h->stream>>>(fa);
}

template <int MODEL, bool OVERLAP>
static void launch_cells(gvizCudaForce *h, const CellArgs &ca, bool count) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (count)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_walk_f32_cells<MODEL, OVERLAP, true>,
                                                  kCellThreads, kCellDyn);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_walk_f32_cells<MODEL, OVERLAP, false>,
                                                  kCellThreads, kCellDyn);
  const uint32_t resident = (uint32_t)((per > 0 ? per : 1) * (sms > 0 ? sms : 1));
  const uint32_t need = blocks(((h->V + 31) / 32) * 32, kCellThreads);
  const uint32_t grid = need < resident ? need : resident;
  cudaMemsetAsync(h->d_groupCount + 1, 0, sizeof(uint32_t), h->stream);
  if (count)
    k_walk_f32_cells<MODEL, OVERLAP, true><<<grid, kCellThreads, kCellDyn, h->stream>>>(ca);
  else
    k_walk_f32_cells<MODEL, OVERLAP, false><<<grid, kCellThreads, kCellDyn, h->stream>>>(ca);
}

// The cell-group walk's per-warp queues exceed the default dynamic shared
// memory of a block; opted in once per process for every instance.
template <int MODEL, bool OVERLAP, bool COUNT>
static void plain_smem_limits() {
  cudaFuncSetAttribute(k_walk_f32<MODEL, OVERLAP, COUNT>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plain_smem(kWalkMaxThreads, kPlainStack));
  cudaFuncSetAttribute(k_walk_f32_queue<MODEL, OVERLAP, COUNT>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plain_smem(kWalkMaxThreads, kPlainStack));
}

void forces_set_smem_limits() {
  plain_smem_limits<GVIZ_CUDA_MODEL_FR, false, false>();
  plain_smem_limits<GVIZ_CUDA_MODEL_FR, false, true>();
  plain_smem_limits<GVIZ_CUDA_MODEL_FR, true, false>();
  plain_smem_limits<GVIZ_CUDA_MODEL_FR, true, true>();
  plain_smem_limits<GVIZ_CUDA_MODEL_LINLOG, false, false>();
  plain_smem_limits<GVIZ_CUDA_MODEL_LINLOG, false, true>();
  plain_smem_limits<GVIZ_CUDA_MODEL_LINLOG, true, false>();
  plain_smem_limits<GVIZ_CUDA_MODEL_LINLOG, true, true>();
  cudaFuncSetAttribute(k_walk_f32_cells<GVIZ_CUDA_MODEL_FR, false, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCellDyn);
  cudaFuncSetAttribute(k_walk_f32_cells<GVIZ_CUDA_MODEL_FR, false, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCellDyn);
  cudaFuncSetAttribute(k_walk_f32_cells<GVIZ_CUDA_MODEL_FR, true, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCellDyn);
  cudaFuncSetAttribute(k_walk_f32_cells<GVIZ_CUDA_MODEL_FR, true, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCellDyn);
  cudaFuncSetAttribute(k_walk_f32_cells<GVIZ_CUDA_MODEL_LINLOG, false, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCellDyn);
  cudaFuncSetAttribute(k_walk_f32_cells<GVIZ_CUDA_MODEL_LINLOG, false, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCellDyn);
  cudaFuncSetAttribute(k_walk_f32_cells<GVIZ_CUDA_MODEL_LINLOG, true, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCellDyn);
  cudaFuncSetAttribute(k_walk_f32_cells<GVIZ_CUDA_MODEL_LINLOG, true, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCellDyn);
}

// The hub targets' plain walk, after the learned walk, on a grid that fills
// the GPU; then their epilogues.
template <int MODEL, bool OVERLAP>
static void launch_far_hubs(gvizCudaForce *h, const FarHubArgs &ha) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_walk_f32_hubs<MODEL, OVERLAP>,
                                                kHubThreads, 0);
  const uint32_t fill = (uint32_t)((per > 0 ? per : 1) * (sms > 0 ? sms : 1));
  const uint32_t need = blocks(h->nFarHubs, kHubThreads / 32);
  cudaMemsetAsync(ha.counter, 0, sizeof(uint32_t), h->stream);
  k_walk_f32_hubs<MODEL, OVERLAP><<<need < fill ? need : fill, kHubThreads, 0, h->stream>>>(ha);
}

static FarHubArgs far_hub_args(gvizCudaForce *h, const WalkArgs &a) {
  FarHubArgs ha;
  ha.w = a;
  ha.hubs = h->d_farHubs;
  ha.counter = h->d_farHubs + h->nFarHubs;
  ha.out = h->d_farHubOut;
  ha.nHubs = h->nFarHubs;
  const double r = h->params.theta / h->params.farHubTheta;
  ha.sizeScale = (float)(r * r);
  return ha;
}

static void enqueue_far_hub_walk(gvizCudaForce *h, const FarHubArgs &ha) {
  const bool ov = h->params.preventOverlap != 0;
  if (h->model == GVIZ_CUDA_MODEL_FR) {
    if (ov) launch_far_hubs<GVIZ_CUDA_MODEL_FR, true>(h, ha);
    else launch_far_hubs<GVIZ_CUDA_MODEL_FR, false>(h, ha);
  } else {
    if (ov) launch_far_hubs<GVIZ_CUDA_MODEL_LINLOG, true>(h, ha);
    else launch_far_hubs<GVIZ_CUDA_MODEL_LINLOG, false>(h, ha);
  }
}

static void enqueue_far_walk(gvizCudaForce *h, const WalkArgs &a, uint64_t *counters);

// The learned walk (see k_walk_f32_far and k_walk_f32_cells), then the hub
// targets' plain walk when params.farHubTargets asks for one, then the hubs'
// epilogues, which replace the learned walk's forces of those vertices. (The
// hub walk on a side stream beside the learned walk was measured slower:
// 7.15 vs 6.90 ms per R-MAT scale-22 step with 16,384 hub targets.)
static void enqueue_far(gvizCudaForce *h, const WalkArgs &a, uint64_t *counters) {
  enqueue_far_walk(h, a, counters);
  if (!(h->nFarHubs > 0 && h->d_farHubs)) return;
  const FarHubArgs ha = far_hub_args(h, a);
  enqueue_far_hub_walk(h, ha);
  prof_mark(h, "bh_walk_hubs");
  k_far_hub_epilogue<<<blocks(h->nFarHubs, 256), 256, 0, h->stream>>>(ha);
}

static void enqueue_far_walk(gvizCudaForce *h, const WalkArgs &a, uint64_t *counters) {
  FarArgs fa;
  fa.w = a;
  fa.cells = h->d_cells;
  fa.leafPre = h->d_leafPre;
  fa.mlp = reinterpret_cast<const MlpDev *>(h->d_mlp);
  fa.spread2 = (float)(h->params.farGroupSpread * h->params.farGroupSpread);
  const bool ov = h->params.preventOverlap != 0;
  const bool count = counters != nullptr;
  if (h->params.farCellGroups) {
    CellArgs ca;
    ca.f = fa;
    ca.groups = h->d_groups;
    ca.kids = h->d_kids;
    ca.stackCap = (h->walkStackCap >= 32 && h->walkStackCap <= (uint32_t)kCellStack)
                      ? h->walkStackCap : (uint32_t)kCellStack;
    ca.nGroups = h->d_groupCount;
    ca.cap = (uint32_t)(h->V ? h->V : 1);
    if (h->model == GVIZ_CUDA_MODEL_FR) {
      if (ov) launch_cells<GVIZ_CUDA_MODEL_FR, true>(h, ca, count);
      else launch_cells<GVIZ_CUDA_MODEL_FR, false>(h, ca, count);
    } else {
      if (ov) launch_cells<GVIZ_CUDA_MODEL_LINLOG, true>(h, ca, count);
      else launch_cells<GVIZ_CUDA_MODEL_LINLOG, false>(h, ca, count);
    }
    prof_mark(h, "bh_walk_f32_learned");
    return;
  }
  if (h->model == GVIZ_CUDA_MODEL_FR) {
    if (ov) launch_far<GVIZ_CUDA_MODEL_FR, true>(h, fa, count);
    else launch_far<GVIZ_CUDA_MODEL_FR, false>(h, fa, count);
  } else {
    if (ov) launch_far<GVIZ_CUDA_MODEL_LINLOG, true>(h, fa, count);
    else launch_far<GVIZ_CUDA_MODEL_LINLOG, false>(h, fa, count);
  }
  prof_mark(h, "bh_walk_f32_learned");
}

// Blocks of `threads` threads that fill the GPU once with the persistent
// walk of this handle's model and overlap setting.
uint32_t walk_resident_blocks(gvizCudaForce *h, uint32_t threads) {
  int dev = 0, sms = 0, per = 0;
  const size_t smem = plain_smem(threads, plain_cap(h));
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const bool ov = h->params.preventOverlap != 0;
  const bool fr = h->model == GVIZ_CUDA_MODEL_FR;
  cudaError_t e;
  if (fr) {
    e = ov ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                 &per, k_walk_f32_queue<GVIZ_CUDA_MODEL_FR, true, false>, threads, smem)
           : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                 &per, k_walk_f32_queue<GVIZ_CUDA_MODEL_FR, false, false>, threads, smem);
  } else {
    e = ov ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                 &per, k_walk_f32_queue<GVIZ_CUDA_MODEL_LINLOG, true, false>, threads, smem)
           : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                 &per, k_walk_f32_queue<GVIZ_CUDA_MODEL_LINLOG, false, false>, threads, smem);
  }
  if (e != cudaSuccess || per <= 0 || sms <= 0) return 0;
  return (uint32_t)(per * sms);
}

void enqueue_walk_f32(gvizCudaForce *h, uint64_t *counters) {
  WalkArgs a;
  a.nodes = reinterpret_cast<const NodeF *>(h->d_nodes);
  a.idx = h->d_idx;
  a.gid = h->d_gid;
  a.active = h->d_active;
  a.graphBase = h->d_graphBase;
  a.rootT = h->d_rootT;
  a.pos = h->d_pos;
  a.massF = h->d_massF;
  a.radiusF = h->d_radiusF;
  a.attF = h->d_attF;
  a.epi = make_epi(h);
  a.num = (float)(h->params.edgeLength * h->params.edgeLength);
  a.overlapC = (float)h->params.overlapConstant;
  a.V = (uint32_t)h->V;
  a.counters = reinterpret_cast<unsigned long long *>(counters);
  a.queue = h->d_walkQueue;
  a.maxNodes = (uint32_t)h->maxNodes;
  a.kids = h->d_kids;
  a.tasks = h->d_walkTasks;
  a.nTasks = h->nWalkTasks;
  a.stackCap = plain_cap(h);
  const bool ov = h->params.preventOverlap != 0;
  const bool fr = h->model == GVIZ_CUDA_MODEL_FR;
  if (h->params.farField && h->d_mlp) {
    enqueue_far(h, a, counters);
    return;
  }
  if (counters) {
    if (fr) {
      if (ov) launch_walk<GVIZ_CUDA_MODEL_FR, true, true>(h, a);
      else launch_walk<GVIZ_CUDA_MODEL_FR, false, true>(h, a);
    } else {
      if (ov) launch_walk<GVIZ_CUDA_MODEL_LINLOG, true, true>(h, a);
      else launch_walk<GVIZ_CUDA_MODEL_LINLOG, false, true>(h, a);
    }
  } else {
    if (fr) {
      if (ov) launch_walk<GVIZ_CUDA_MODEL_FR, true, false>(h, a);
      else launch_walk<GVIZ_CUDA_MODEL_FR, false, false>(h, a);
    } else {
      if (ov) launch_walk<GVIZ_CUDA_MODEL_LINLOG, true, false>(h, a);
      else launch_walk<GVIZ_CUDA_MODEL_LINLOG, false, false>(h, a);
    }
  }
  prof_mark(h, "bh_walk_f32");
}

// Source ranges of the exact FP32 kernel for V vertices on a GPU of `sms`
// SMs: enough blocks for about four waves, at least four tiles per range.
uint32_t exact_splits(size_t V, int sms) {
  const size_t tb = (V + kExactThreads * kExactTpt - 1) / (kExactThreads * kExactTpt);
  if (tb == 0) return 1;
  size_t s = (4 * (size_t)(sms > 0 ? sms : 1) + tb - 1) / tb;
  s = std::min<size_t>(s, (V + 4 * kExactTile - 1) / (4 * kExactTile));
  return (uint32_t)std::max<size_t>(1, std::min<size_t>(s, 32));
}

void enqueue_exact_f32(gvizCudaForce *h) {
  ExactArgs a;
  a.pos = h->d_pos;
  a.massF = h->d_massF;
  a.radiusF = h->d_radiusF;
  a.gid = h->d_gid;
  a.active = h->d_active;
  a.graphOff = h->d_graphOff;
  a.attF = h->d_attF;
  a.epi = make_epi(h);
  a.num = (float)(h->params.edgeLength * h->params.edgeLength);
  a.overlapC = (float)h->params.overlapConstant;
  a.V = (uint32_t)h->V;
  a.partial = h->d_exactPartial;
  a.splits = h->d_exactPartial ? h->exactSplits : 1u;
  const dim3 grid(blocks(h->V, kExactThreads * kExactTpt), a.splits);
  const bool ov = h->params.preventOverlap != 0;
  if (h->model == GVIZ_CUDA_MODEL_FR) {
    if (ov) k_exact_f32<GVIZ_CUDA_MODEL_FR, true><<<grid, kExactThreads, 0, h->stream>>>(a);
    else k_exact_f32<GVIZ_CUDA_MODEL_FR, false><<<grid, kExactThreads, 0, h->stream>>>(a);
  } else {
    if (ov) k_exact_f32<GVIZ_CUDA_MODEL_LINLOG, true><<<grid, kExactThreads, 0, h->stream>>>(a);
    else k_exact_f32<GVIZ_CUDA_MODEL_LINLOG, false><<<grid, kExactThreads, 0, h->stream>>>(a);
  }
  if (a.splits > 1) k_exact_combine<<<blocks(h->V, 256), 256, 0, h->stream>>>(a);
  prof_mark(h, "exact_f32");
}
