// precise.cu -- FP64 force kernels and the ForceAtlas2 speed / update
// kernels. This translation unit is compiled with --fmad=false so every
// a*b+c rounds twice, exactly like the reference's C (x86-64, no FMA):
// with the same inputs and the same order of terms the FP64 walk, the FP64
// exact kernel and the FA2 arithmetic reproduce the reference's rounding.
//
//  * k_attr_f64  : src/embedders/gvizForceEmbedder.c:93-100 in CSR order
//  * k_walk_f64  : bhAccumulateRepulsion (:35-74), warp-shared traversal as in
//                  forces.cu, terms summed in the reference's DFS order
//  * k_exact_f64 : the BH-off loop (:104-115), j ascending, j != i
//  * k_fa2_*     : swing/traction sums, updateGlobalSpeed (:140-185),
//                  applySpeedRange (:187-197), step tail (:467-492)
#include <math.h>

#include "epilogue.cuh"
#include "internal.cuh"

int dir_table_upload_precise(const double *t) {
  return cudaMemcpyToSymbol(c_dirTable, t, sizeof(double) * 2 * GVIZ_DIR_TABLE) ==
                 cudaSuccess ? 0 : -1;
}

EpiArgs make_epi(gvizCudaForce *h) {
  EpiArgs e;
  e.pos = h->d_pos;
  e.degree = h->d_degree;
  e.mass = h->d_mass;
  e.sf = h->forceOnly ? h->d_applied : h->d_sf;
  e.sfOld = h->d_sfOld;
  e.disp = h->d_disp;
  e.att = h->d_att;
  e.rep = h->d_rep;
  e.swing = h->d_swing;
  e.trac = h->d_trac;
  e.repVec = h->repVecOut;
  e.gravityK = h->params.gravityK;
  return e;
}

namespace {

constexpr int kThreads = 256;
constexpr int kWalkThreads = 128;
constexpr int kExactTile = 256;
constexpr uint32_t kInf = 0xffffffffu;

struct Attr64Args {
  const uint32_t *rowOff, *cols, *gid, *active;
  const double2 *pos;
  double2 *out;
  double k;
  uint32_t V;
};

template <int MODEL>
__global__ __launch_bounds__(kThreads) void k_attr_f64(Attr64Args a) {
  const uint32_t v = blockIdx.x * kThreads + threadIdx.x;
  if (v >= a.V) return;
  if (a.active && !a.active[a.gid ? a.gid[v] : 0u]) return;
  const double2 p = a.pos[v];
  double ax = 0.0, ay = 0.0;
  const uint32_t e1 = a.rowOff[v + 1];
  for (uint32_t e = a.rowOff[v]; e < e1; e++) {
    const double2 q = a.pos[a.cols[e]];
    const double dx = q.x - p.x;
    const double dy = q.y - p.y;
    const double dist = sqrt(dx * dx + dy * dy);
    if (dist < 1e-9) continue;
    double s;
    if (MODEL == GVIZ_CUDA_MODEL_FR)
      s = dist / a.k;
    else
      s = log(1.0 + dist) / dist;
    ax += s * dx;
    ay += s * dy;
  }
  a.out[v] = make_double2(ax, ay);
}

// FR / LinLog repulsion term added to (ax, ay) with the reference's
// operation order (include/core/gvizVec.h:404-428, 552-578;
// src/embedders/gvizForceDirected.c:141-149 for FR's mass * force).
template <int MODEL>
__device__ __forceinline__ void rep_term64(double vx, double vy, double ux,
                                           double uy, double vMass,
                                           double oMass, double radiusSum,
                                           double kk, double C, uint32_t self,
                                           uint32_t other, double &ax,
                                           double &ay) {
  const double dx = ux - vx;
  const double dy = uy - vy;
  const double distSq = dx * dx + dy * dy;
  const double dist = sqrt(distSq);
  const double gap = dist - radiusSum;
  const double num = (MODEL == GVIZ_CUDA_MODEL_FR) ? kk : vMass * oMass;
  const double mag = gap > 0.0 ? num / gap : num * C;
  double dirx, diry;
  if (dist > 0.0) {
    dirx = dx / dist;
    diry = dy / dist;
  } else {
    coincident_dir(self, other, dirx, diry);
  }
  if (MODEL == GVIZ_CUDA_MODEL_FR) {
    const double sx = 0.0 - mag * dirx;
    const double sy = 0.0 - mag * diry;
    const double m = (double)(unsigned long long)oMass;
    ax += m * sx;
    ay += m * sy;
  } else {
    ax -= mag * dirx;
    ay -= mag * diry;
  }
}

struct Walk64Args {
  const NodeD *nodes;
  const uint32_t *idx, *gid, *active, *graphBase, *rootT;
  const double2 *pos;
  const double *mass, *radius;
  const double2 *attD;
  EpiArgs epi;
  double kk, overlapC, theta;
  uint32_t V, maxNodes;
};

template <int MODEL>
__global__ __launch_bounds__(kWalkThreads) void k_walk_f64(Walk64Args a) {
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t s = ((blockIdx.x * kWalkThreads + threadIdx.x) >> 5) * 32u + lane;
  const bool valid = s < a.V;
  const uint32_t v = valid ? a.idx[s] : 0u;
  const uint32_t g = (valid && a.gid) ? a.gid[v] : 0u;
  const bool act = valid && (a.active == nullptr || a.active[g] != 0u);
  uint32_t resume = 0, myEnd = 0;
  double vx = 0.0, vy = 0.0, mv = 0.0, rv = 0.0;
  if (act) {
    resume = a.graphBase[g];
    myEnd = min(resume + a.rootT[g], a.maxNodes);
    const double2 p = a.pos[v];
    vx = p.x;
    vy = p.y;
    mv = a.mass[v];
    rv = a.radius[v];
  }
  double ax = 0.0, ay = 0.0;
  uint32_t nxt = resume < myEnd ? resume : kInf;
  uint32_t cur = __reduce_min_sync(0xffffffffu, nxt);
  while (cur != kInf) {
    const double2 n0 = __ldg(reinterpret_cast<const double2 *>(a.nodes + cur));
    const double2 n1 = __ldg(reinterpret_cast<const double2 *>(a.nodes + cur) + 1);
    const int4 n2 = __ldg(reinterpret_cast<const int4 *>(a.nodes + cur) + 2);
    const bool active = cur >= resume && cur < myEnd;
    const bool isLeaf = n2.y >= 0;
    const bool massOk = n1.x != 0.0;
    bool open = false;
    if (active && massOk) {
      if (isLeaf) {
        if ((uint32_t)n2.y != v)
          rep_term64<MODEL>(vx, vy, n0.x, n0.y, mv, n1.x, rv + n1.y, a.kk,
                            a.overlapC, v, (uint32_t)n2.y, ax, ay);
      } else {
        const double dx = n0.x - vx;
        const double dy = n0.y - vy;
        const double dist = sqrt(dx * dx + dy * dy);
        const double ratio = (2.0 * n1.y) / dist;
        if (ratio < a.theta)
          rep_term64<MODEL>(vx, vy, n0.x, n0.y, mv, n1.x, rv, a.kk,
                            a.overlapC, v, v, ax, ay);
        else
          open = true;
      }
    }
    if (active) resume = open ? cur + 1u : max((uint32_t)n2.x, cur + 1u);
    nxt = resume < myEnd ? resume : kInf;
    cur = __reduce_min_sync(0xffffffffu, nxt);
  }
  if (!act) return;
  const double2 at = a.attD[v];
  force_epilogue(a.epi, v, at.x, at.y, ax, ay);
}

struct Exact64Args {
  const double2 *pos;
  const double *mass, *radius;
  const uint32_t *gid, *active, *targets;
  const uint64_t *graphOff;
  const double2 *attD;
  EpiArgs epi;
  double2 *judgeOut;  // target-list mode: repulsion vectors only
  double kk, overlapC;
  uint32_t n;         // number of targets (V, or the list length)
};

template <int MODEL>
__global__ __launch_bounds__(kThreads) void k_exact_f64(Exact64Args a) {
  __shared__ double2 sp[kExactTile];
  __shared__ double2 smr[kExactTile];
  __shared__ uint32_t sRange[2];
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  const bool valid = t < a.n;
  const uint32_t v = valid ? (a.targets ? a.targets[t] : t) : 0u;
  const uint32_t g = (valid && a.gid) ? a.gid[v] : 0u;
  const bool act = valid && (a.targets || a.active == nullptr || a.active[g] != 0u);
  uint32_t gb = 0, ge = 0;
  if (act) {
    gb = (uint32_t)a.graphOff[g];
    ge = (uint32_t)a.graphOff[g + 1];
  }
  if (threadIdx.x == 0) {
    sRange[0] = kInf;
    sRange[1] = 0;
  }
  __syncthreads();
  if (act) {
    atomicMin(&sRange[0], gb);
    atomicMax(&sRange[1], ge);
  }
  __syncthreads();
  const uint32_t lo = sRange[0], hi = sRange[1];
  double vx = 0.0, vy = 0.0, mv = 0.0, rv = 0.0;
  if (act) {
    const double2 p = a.pos[v];
    vx = p.x;
    vy = p.y;
    mv = a.mass[v];
    rv = a.radius[v];
  }
  double ax = 0.0, ay = 0.0;
  for (uint32_t t0 = lo; t0 < hi; t0 += kExactTile) {
    __syncthreads();
    const uint32_t j = t0 + threadIdx.x;
    if (threadIdx.x < kExactTile && j < hi) {
      sp[threadIdx.x] = a.pos[j];
      smr[threadIdx.x] = make_double2(a.mass[j], a.radius[j]);
    }
    __syncthreads();
    const uint32_t cnt = min((uint32_t)kExactTile, hi - t0);
    if (act) {
      for (uint32_t q = 0; q < cnt; q++) {
        const uint32_t jj = t0 + q;
        if (jj == v || jj < gb || jj >= ge) continue;
        const double2 u = sp[q];
        const double2 mr = smr[q];
        rep_term64<MODEL>(vx, vy, u.x, u.y, mv, mr.x, rv + mr.y, a.kk,
                          a.overlapC, v, jj, ax, ay);
      }
    }
  }
  if (!act) return;
  if (a.judgeOut) {
    a.judgeOut[t] = make_double2(ax, ay);
    return;
  }
  const double2 at = a.attD[v];
  force_epilogue(a.epi, v, at.x, at.y, ax, ay);
}

// ---------------------------------------------------------------------------
// ForceAtlas2 speed regulation and the position update
// ---------------------------------------------------------------------------

struct Fa2Args {
  const uint32_t *chunkBegin, *chunkEnd, *chunkGraph, *gChunkBegin,
      *gChunkEnd;
  const uint64_t *graphOff;
  const double *swing, *trac, *att, *rep, *meanDegPlusOne;
  const double2 *disp;
  double2 *pos, *applied;
  ChunkStat *chunkStat;
  double *speed, *eff, *stats, *lastStats;
  uint32_t *active, *anyActive;
  uint64_t *iter, *runLeft;
  const double *runEps;
  double jitterTolerance, gravityK;
  uint32_t G;
  int strict;
};

// Fixed-shape block sum: strided per-thread partials, xor-shuffle tree,
// warp partials added in warp order. Same inputs -> same bits.
__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31u) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kThreads / 32; w++) r += sh[w];
  __syncthreads();
  return r;
}

__device__ __forceinline__ double block_max(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31u) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kThreads / 32; w++) r = fmax(r, sh[w]);
  __syncthreads();
  return r;
}

__global__ __launch_bounds__(kThreads) void k_fa2_chunks(Fa2Args a) {
  __shared__ double sh[kThreads / 32];
  const uint32_t c = blockIdx.x;
  const uint32_t g = a.chunkGraph[c];
  if (!a.active[g]) return;
  double sw = 0.0, tr = 0.0;
  for (uint32_t v = a.chunkBegin[c] + threadIdx.x; v < a.chunkEnd[c]; v += kThreads) {
    sw += a.swing[v];
    tr += a.trac[v];
  }
  sw = block_sum(sw, sh);
  tr = block_sum(tr, sh);
  if (threadIdx.x == 0) {
    a.chunkStat[c].a = sw;
    a.chunkStat[c].b = tr;
  }
}

// updateGlobalSpeed, src/embedders/gvizForceEmbedder.c:140-185, per graph
// One block per graph; thread 0 applies the rule to the block's sums.
__global__ __launch_bounds__(kThreads) void k_fa2_speed(Fa2Args a) {
  __shared__ double sh[kThreads / 32];
  const uint32_t g = blockIdx.x;
  if (!a.active[g]) return;
  double totalSwing = 0.0, totalTraction = 0.0;
  if (a.strict) {
    if (threadIdx.x == 0)
      for (uint64_t v = a.graphOff[g]; v < a.graphOff[g + 1]; v++) {
        totalSwing += a.swing[v];
        totalTraction += a.trac[v];
      }
  } else {
    for (uint32_t c = a.gChunkBegin[g] + threadIdx.x; c < a.gChunkEnd[g]; c += kThreads) {
      totalSwing += a.chunkStat[c].a;
      totalTraction += a.chunkStat[c].b;
    }
    totalSwing = block_sum(totalSwing, sh);
    totalTraction = block_sum(totalTraction, sh);
  }
  if (threadIdx.x != 0) return;
  if (totalTraction < 1e-7) return;
  double speed = a.speed[g], eff = a.eff[g];
  const double n = (double)(a.graphOff[g + 1] - a.graphOff[g]);
  const double estimatedOptimalJT = 0.05 * sqrt(n);
  const double minJT = sqrt(estimatedOptimalJT);
  const double maxJT = 10.0;
  double jt = a.jitterTolerance *
              fmax(minJT, fmin(maxJT, estimatedOptimalJT * totalTraction / (n * n)));
  if (totalSwing / totalTraction > 2.0) {
    if (eff > 0.05) eff *= 0.5;
    jt = fmax(jt, a.jitterTolerance);
  }
  const double targetSpeed =
      totalSwing > 1e-7 ? jt * eff * totalTraction / totalSwing : speed;
  if (totalSwing > jt * totalTraction) {
    if (eff > 0.05) eff *= 0.7;
  } else if (speed < 1000.0) {
    eff *= 1.3;
  }
  if (eff < 0.05)
    eff = 0.05;
  else if (eff > 1.0)
    eff = 1.0;
  speed += fmin(targetSpeed - speed, 0.5 * speed);
  a.speed[g] = speed;
  a.eff[g] = eff;
}

// applySpeedRange (:187-197) + position update and stat partials (:467-477)
__global__ __launch_bounds__(kThreads) void k_fa2_apply(Fa2Args a) {
  __shared__ double sh[kThreads / 32];
  const uint32_t c = blockIdx.x;
  const uint32_t g = a.chunkGraph[c];
  if (!a.active[g]) return;
  const double speed = a.speed[g];
  double mx = 0.0, sAtt = 0.0, sRep = 0.0;
  for (uint32_t v = a.chunkBegin[c] + threadIdx.x; v < a.chunkEnd[c]; v += kThreads) {
    const double factor = speed / (1.0 + sqrt(speed * a.swing[v]));
    const double2 f = a.disp[v];
    const double2 o = make_double2(f.x * factor, f.y * factor);
    a.applied[v] = o;
    const double nrm = sqrt(o.x * o.x + o.y * o.y);
    mx = fmax(mx, nrm);
    sAtt += a.att[v];
    sRep += a.rep[v];
    double2 p = a.pos[v];
    p.x += o.x;
    p.y += o.y;
    a.pos[v] = p;
  }
  mx = block_max(mx, sh);
  sAtt = block_sum(sAtt, sh);
  sRep = block_sum(sRep, sh);
  if (threadIdx.x == 0) {
    a.chunkStat[c].a = mx;
    a.chunkStat[c].b = sAtt;
    a.chunkStat[c].c = sRep;
  }
}

__global__ __launch_bounds__(kThreads) void k_fa2_stats(Fa2Args a) {
  __shared__ double sh[kThreads / 32];
  const uint32_t g = blockIdx.x;
  if (!a.active[g]) return;
  double mx = 0.0, sAtt = 0.0, sRep = 0.0;
  if (a.strict) {
    if (threadIdx.x == 0)
      for (uint64_t v = a.graphOff[g]; v < a.graphOff[g + 1]; v++) {
        const double2 o = a.applied[v];
        const double nrm = sqrt(o.x * o.x + o.y * o.y);
        if (nrm > mx) mx = nrm;
        sAtt += a.att[v];
        sRep += a.rep[v];
      }
  } else {
    for (uint32_t c = a.gChunkBegin[g] + threadIdx.x; c < a.gChunkEnd[g]; c += kThreads) {
      mx = fmax(mx, a.chunkStat[c].a);
      sAtt += a.chunkStat[c].b;
      sRep += a.chunkStat[c].c;
    }
    mx = block_max(mx, sh);
    sAtt = block_sum(sAtt, sh);
    sRep = block_sum(sRep, sh);
  }
  if (threadIdx.x != 0) return;
  const uint64_t n = a.graphOff[g + 1] - a.graphOff[g];
  const uint64_t it = a.iter[g];
  double *row = a.stats + ((it % GVIZ_STATS_CAP) * a.G + g) * 5;
  row[0] = mx;
  row[1] = a.speed[g];
  row[2] = n ? sAtt / (double)n : 0.0;
  row[3] = n ? sRep / (double)n : 0.0;
  row[4] = a.gravityK * a.meanDegPlusOne[g];
  for (int q = 0; q < 5; q++) a.lastStats[5 * g + q] = row[q];
  a.iter[g] = it + 1;
  const uint64_t left = a.runLeft[g] - 1;
  a.runLeft[g] = left;
  if (mx < a.runEps[g] || left == 0) {
    a.active[g] = 0;
    atomicSub(a.anyActive, 1u);
  }
}

inline uint32_t blocks(size_t n, int t) { return (uint32_t)((n + t - 1) / t); }

Fa2Args make_fa2(gvizCudaForce *h) {
  Fa2Args a;
  a.chunkBegin = h->d_chunkBegin;
  a.chunkEnd = h->d_chunkEnd;
  a.chunkGraph = h->d_chunkGraph;
  a.gChunkBegin = h->d_gChunkBegin;
  a.gChunkEnd = h->d_gChunkEnd;
  a.graphOff = h->d_graphOff;
  a.swing = h->d_swing;
  a.trac = h->d_trac;
  a.att = h->d_att;
  a.rep = h->d_rep;
  a.meanDegPlusOne = h->d_meanDegPlusOne;
  a.disp = h->d_disp;
  a.pos = h->d_pos;
  a.applied = h->d_applied;
  a.chunkStat = h->d_chunkStat;
  a.speed = h->d_speed;
  a.eff = h->d_eff;
  a.stats = h->d_stats;
  a.lastStats = h->d_lastStats;
  a.active = h->d_active;
  a.anyActive = h->d_anyActive;
  a.iter = h->d_iter;
  a.runLeft = h->d_runLeft;
  a.runEps = h->d_runEps;
  a.jitterTolerance = h->params.jitterTolerance;
  a.gravityK = h->params.gravityK;
  a.G = (uint32_t)h->G;
  a.strict = h->params.strictReductions;
  return a;
}

Exact64Args make_exact64(gvizCudaForce *h) {
  Exact64Args a;
  a.pos = h->d_pos;
  a.mass = h->d_mass;
  a.radius = h->d_radius;
  a.gid = h->d_gid;
  a.active = h->d_active;
  a.targets = nullptr;
  a.graphOff = h->d_graphOff;
  a.attD = h->d_attD;
  a.epi = make_epi(h);
  a.judgeOut = nullptr;
  a.kk = h->params.edgeLength * h->params.edgeLength;
  a.overlapC = h->params.overlapConstant;
  a.n = (uint32_t)h->V;
  return a;
}

}  // namespace

void enqueue_attraction_f64(gvizCudaForce *h) {
  Attr64Args a;
  a.rowOff = h->d_rowOff;
  a.cols = h->d_cols;
  a.gid = h->d_gid;
  a.active = h->d_active;
  a.pos = h->d_pos;
  a.out = h->d_attD;
  a.k = h->params.edgeLength;
  a.V = (uint32_t)h->V;
  if (h->model == GVIZ_CUDA_MODEL_FR)
    k_attr_f64<GVIZ_CUDA_MODEL_FR><<<blocks(h->V, kThreads), kThreads, 0, h->stream>>>(a);
  else
    k_attr_f64<GVIZ_CUDA_MODEL_LINLOG><<<blocks(h->V, kThreads), kThreads, 0, h->stream>>>(a);
  prof_mark(h, "attraction_f64");
}

void enqueue_walk_f64(gvizCudaForce *h) {
  Walk64Args a;
  a.nodes = reinterpret_cast<const NodeD *>(h->d_nodes);
  a.idx = h->d_idx;
  a.gid = h->d_gid;
  a.active = h->d_active;
  a.graphBase = h->d_graphBase;
  a.rootT = h->d_rootT;
  a.pos = h->d_pos;
  a.mass = h->d_mass;
  a.radius = h->d_radius;
  a.attD = h->d_attD;
  a.epi = make_epi(h);
  a.kk = h->params.edgeLength * h->params.edgeLength;
  a.overlapC = h->params.overlapConstant;
  a.theta = h->params.theta;
  a.V = (uint32_t)h->V;
  a.maxNodes = (uint32_t)h->maxNodes;
  const uint32_t grid = blocks(((h->V + 31) / 32) * 32, kWalkThreads);
  if (h->model == GVIZ_CUDA_MODEL_FR)
    k_walk_f64<GVIZ_CUDA_MODEL_FR><<<grid, kWalkThreads, 0, h->stream>>>(a);
  else
    k_walk_f64<GVIZ_CUDA_MODEL_LINLOG><<<grid, kWalkThreads, 0, h->stream>>>(a);
  prof_mark(h, "bh_walk_f64");
}

void enqueue_exact_f64(gvizCudaForce *h) {
  Exact64Args a = make_exact64(h);
  if (h->model == GVIZ_CUDA_MODEL_FR)
    k_exact_f64<GVIZ_CUDA_MODEL_FR><<<blocks(h->V, kThreads), kThreads, 0, h->stream>>>(a);
  else
    k_exact_f64<GVIZ_CUDA_MODEL_LINLOG><<<blocks(h->V, kThreads), kThreads, 0, h->stream>>>(a);
  prof_mark(h, "exact_f64");
}

void enqueue_exact_judge(gvizCudaForce *h, const uint32_t *d_targets, size_t n,
                         double2 *d_out) {
  Exact64Args a = make_exact64(h);
  a.targets = d_targets;
  a.judgeOut = d_out;
  a.n = (uint32_t)n;
  if (h->model == GVIZ_CUDA_MODEL_FR)
    k_exact_f64<GVIZ_CUDA_MODEL_FR><<<blocks(n, kThreads), kThreads, 0, h->stream>>>(a);
  else
    k_exact_f64<GVIZ_CUDA_MODEL_LINLOG><<<blocks(n, kThreads), kThreads, 0, h->stream>>>(a);
}

void enqueue_fa2(gvizCudaForce *h) {
  Fa2Args a = make_fa2(h);
  const uint32_t G = (uint32_t)h->G;
  if (!h->params.strictReductions)
    k_fa2_chunks<<<h->nChunks, kThreads, 0, h->stream>>>(a);
  k_fa2_speed<<<G, kThreads, 0, h->stream>>>(a);
  k_fa2_apply<<<h->nChunks, kThreads, 0, h->stream>>>(a);
  k_fa2_stats<<<G, kThreads, 0, h->stream>>>(a);
  prof_mark(h, "fa2_update");
}
