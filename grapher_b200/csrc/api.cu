// api.cu -- the C ABI of libgvizcuda (include/gvizcuda.h).
//
// One handle = one set of device buffers + one stream. A step is
//   structForce -> oldStructForce            (gvizForceEmbedder.c:449-450)
//   quadtree rebuild (tree.cu)               (:451-453)
//   attraction + repulsion + gravity         (:455-457, computeForceRange)
//   swing/traction, global speed, apply      (:459-465)
//   step tail and the five stats             (:467-492)
// captured once into a CUDA graph and replayed; nothing in it waits on the
// host, so Run() can enqueue many steps and check convergence in batches.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "epilogue.cuh"
#include "internal.cuh"

void tree_set_smem_limits();
void sort_set_smem_limits();
void enqueue_cell_dump(gvizCudaForce *h, int32_t *depth, uint64_t *hi,
                       uint64_t *lo, double *mass, double *cx, double *cy,
                       uint64_t *cnt);

static int far_judge(gvizCudaForce *h);

namespace {

constexpr int kRunBatch = 8;

int set_err(gvizCudaForce *h, int code) {
  if (h && code != GVIZ_CUDA_OK) h->lastError = code;
  return code;
}

template <typename T>
int dalloc(gvizCudaForce *h, T **p, size_t count) {
  size_t bytes = count * sizeof(T);
  if (bytes == 0) bytes = 16;
  if (cudaMalloc((void **)p, bytes) != cudaSuccess) {
    *p = nullptr;
    return set_err(h, GVIZ_CUDA_ERR_ALLOC);
  }
  return GVIZ_CUDA_OK;
}

template <typename T>
void dfree(T *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}

bool g_dirUploaded[64] = {false};

int upload_dir_table(gvizCudaForce *h) {
  if (h->device < 64 && g_dirUploaded[h->device]) return GVIZ_CUDA_OK;
  double t[2 * GVIZ_DIR_TABLE];
  for (int k = 0; k < GVIZ_DIR_TABLE; k++) {
    double a = 2.0 * M_PI * (double)k / (double)GVIZ_DIR_TABLE;
    t[2 * k] = cos(a);
    t[2 * k + 1] = sin(a);
  }
  if (dir_table_upload_forces(t) || dir_table_upload_precise(t))
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  if (h->device < 64) g_dirUploaded[h->device] = true;
  return GVIZ_CUDA_OK;
}

void free_all(gvizCudaForce *h) {
  dfree(h->d_judgeIdx);
  dfree(h->d_judgeExact);
  dfree(h->d_judgeOut);
  dfree(h->d_judgeRep);
  dfree(h->d_rowOff);
  dfree(h->d_cols);
  dfree(h->d_degree);
  dfree(h->d_mass);
  dfree(h->d_massF);
  dfree(h->d_radius);
  dfree(h->d_radiusF);
  dfree(h->d_gid);
  dfree(h->d_graphOff);
  dfree(h->d_meanDegPlusOne);
  dfree(h->d_chunkBegin);
  dfree(h->d_chunkEnd);
  dfree(h->d_chunkGraph);
  dfree(h->d_gChunkBegin);
  dfree(h->d_gChunkEnd);
  dfree(h->d_attrLight);
  dfree(h->d_attrHeavy);
  dfree(h->d_hubV);
  dfree(h->d_hubFirst);
  dfree(h->d_hubChunkV);
  dfree(h->d_hubChunkE0);
  dfree(h->d_hubChunkE1);
  dfree(h->d_hubPartial);
  dfree(h->d_pos);
  dfree(h->d_sf);
  dfree(h->d_sfOld);
  dfree(h->d_disp);
  dfree(h->d_applied);
  dfree(h->d_att);
  dfree(h->d_rep);
  dfree(h->d_swing);
  dfree(h->d_trac);
  dfree(h->d_attF);
  dfree(h->d_attD);
  dfree(h->d_speed);
  dfree(h->d_eff);
  dfree(h->d_active);
  dfree(h->d_anyActive);
  dfree(h->d_iter);
  dfree(h->d_runLeft);
  dfree(h->d_runEps);
  dfree(h->d_stats);
  dfree(h->d_lastStats);
  dfree(h->d_chunkStat);
  dfree(h->d_status);
  dfree(h->d_chunkBox);
  dfree(h->d_roots);
  dfree(h->d_keyHi);
  dfree(h->d_keyLo);
  dfree(h->d_ck);
  dfree(h->d_ckAlt);
  dfree(h->d_idx);
  dfree(h->d_idxAlt);
  dfree(h->d_sHi);
  dfree(h->d_sLo);
  dfree(h->d_flag);
  dfree(h->d_scan);
  dfree(h->d_deepRuns);
  dfree(h->d_counts);
  dfree(h->d_sortState);
  dfree(h->d_scanState);
  dfree(h->d_bHi);
  dfree(h->d_bLo);
  dfree(h->d_bGid);
  dfree(h->d_bStart);
  dfree(h->d_nLeft);
  dfree(h->d_nRight);
  dfree(h->d_nFirst);
  dfree(h->d_nLast);
  dfree(h->d_nDelta);
  dfree(h->d_nCounter);
  dfree(h->d_upInt);
  dfree(h->d_upLeaf);
  dfree(h->d_nM);
  dfree(h->d_nSX);
  dfree(h->d_nSY);
  dfree(h->d_nCnt);
  dfree(h->d_nT);
  dfree(h->d_nFlag);
  dfree(h->d_bM);
  dfree(h->d_bSX);
  dfree(h->d_bSY);
  dfree(h->d_bCnt);
  dfree(h->d_bT);
  dfree(h->d_rootNode);
  dfree(h->d_rootT);
  dfree(h->d_graphBase);
  dfree(h->d_nodes);
  dfree(h->d_kids);
  dfree(h->d_exactPartial);
  dfree(h->d_leafDepth);
  dfree(h->d_counters);
  dfree(h->d_walkQueue);
  dfree(h->d_walkTasks);
}

int upload_radius(gvizCudaForce *h) {
  const size_t V = h->V;
  std::vector<double> r(V ? V : 1, 0.0);
  std::vector<float> rf(V ? V : 1, 0.0f);
  std::vector<uint32_t> deg(V ? V : 1);
  if (V && cudaMemcpy(deg.data(), h->d_degree, V * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  if (h->params.preventOverlap) {
    // gvizForceEmbedderVertexRadius, src/embedders/gvizForceEmbedder.c:389-393
    for (size_t i = 0; i < V; i++) {
      r[i] = h->params.radiusBase *
             (1.0 + h->params.radiusPerDegree * sqrt((double)deg[i]));
      rf[i] = (float)r[i];
    }
  }
  if (V && (cudaMemcpy(h->d_radius, r.data(), V * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(h->d_radiusF, rf.data(), V * 4, cudaMemcpyHostToDevice) != cudaSuccess))
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  return GVIZ_CUDA_OK;
}

// ---- the step ------------------------------------------------------------

void enqueue_step(gvizCudaForce *h) {
  cudaStream_t st = h->stream;
  cudaMemsetAsync(h->d_status, 0, sizeof(uint32_t), st);
  cudaMemcpyAsync(h->d_sfOld, h->d_sf, h->V * sizeof(double2),
                  cudaMemcpyDeviceToDevice, st);
  const bool f64 = h->params.precision == GVIZ_CUDA_FP64;
  const bool bh = h->params.barnesHutEnabled != 0;
  // attraction reads positions only and its forces are first read by the
  // repulsion pass: with a tree to build it runs on the side stream,
  // overlapping the build (in order while profiling, so that each kernel
  // keeps its own time)
  const bool overlap = bh && h->side && !h->profiling;
  if (overlap) {
    cudaEventRecord(h->evFork, st);
    cudaStreamWaitEvent(h->side, h->evFork, 0);
    h->stream = h->side;
    if (f64)
      enqueue_attraction_f64(h);
    else
      enqueue_attraction_f32(h);
    h->stream = st;
    cudaEventRecord(h->evJoin, h->side);
    enqueue_tree_build(h);
    cudaStreamWaitEvent(st, h->evJoin, 0);
  } else {
    if (bh) enqueue_tree_build(h);
    if (f64)
      enqueue_attraction_f64(h);
    else
      enqueue_attraction_f32(h);
  }
  if (bh) {
    if (f64)
      enqueue_walk_f64(h);
    else
      enqueue_walk_f32(h, nullptr);
  } else {
    if (f64)
      enqueue_exact_f64(h);
    else
      enqueue_exact_f32(h);
  }
  if (!h->forceOnly) enqueue_fa2(h);
}

int ensure_graph(gvizCudaForce *h) {
  if (!h->graphDirty && h->stepExec) return GVIZ_CUDA_OK;
  if (h->stepExec) {
    cudaGraphExecDestroy(h->stepExec);
    h->stepExec = nullptr;
  }
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  enqueue_step(h);
  if (cudaStreamEndCapture(h->stream, &g) != cudaSuccess || !g)
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  size_t nNodes = 0;
  cudaGraphGetNodes(g, nullptr, &nNodes);
  std::vector<cudaGraphNode_t> nodes(nNodes);
  if (nNodes) cudaGraphGetNodes(g, nodes.data(), &nNodes);
  h->kernelsPerStep = 0;
  for (size_t i = 0; i < nNodes; i++) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
      h->kernelsPerStep++;
  }
  cudaError_t e = cudaGraphInstantiate(&h->stepExec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return set_err(h, GVIZ_CUDA_ERR_CUDA);
  h->graphDirty = false;
  return GVIZ_CUDA_OK;
}

// Replays the captured step n times. With automatic checks of the learned
// walk on (gvizCudaForceSetFarJudge), a check runs before every judgeEvery-th
// step launched while the learned walk is on; a check that turns the walk
// off makes the next replay capture the plain step.
int launch_steps(gvizCudaForce *h, uint32_t n) {
  if (h->V == 0) return GVIZ_CUDA_OK;
  int rc = ensure_graph(h);
  if (rc) return rc;
  for (uint32_t i = 0; i < n; i++) {
    if (h->judgeEvery && h->params.farField && h->d_mlp &&
        h->stepsLaunched >= h->judgeNextAt) {
      rc = far_judge(h);
      if (rc) return rc;
      h->judgeNextAt = h->stepsLaunched + h->judgeEvery;
      rc = ensure_graph(h);
      if (rc) return rc;
    }
    if (cudaGraphLaunch(h->stepExec, h->stream) != cudaSuccess)
      return set_err(h, GVIZ_CUDA_ERR_CUDA);
    h->stepsLaunched++;
  }
  return GVIZ_CUDA_OK;
}

int status_to_code(uint32_t st) {
  if (st & GVIZ_ST_NONFINITE) return GVIZ_CUDA_ERR_NONFINITE;
  if (st & GVIZ_ST_DEEP_RUN) return GVIZ_CUDA_ERR_DEEP_RUN;
  if (st & GVIZ_ST_TREE) return GVIZ_CUDA_ERR_CUDA;
  return GVIZ_CUDA_OK;
}

int sync_and_check(gvizCudaForce *h) {
  if (cudaStreamSynchronize(h->stream) != cudaSuccess)
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  uint32_t st = 0;
  if (cudaMemcpy(&st, h->d_status, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  return set_err(h, status_to_code(st));
}

void set_all_active(gvizCudaForce *h, uint64_t runLeft, double eps) {
  std::vector<uint32_t> one(h->G, 1u);
  std::vector<uint64_t> left(h->G, runLeft);
  std::vector<double> e(h->G, eps);
  uint32_t any = (uint32_t)h->G;
  cudaMemcpy(h->d_active, one.data(), h->G * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(h->d_runLeft, left.data(), h->G * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(h->d_runEps, e.data(), h->G * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(h->d_anyActive, &any, 4, cudaMemcpyHostToDevice);
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

double fill_stats(gvizCudaForce *h, gvizCudaStepStats *stats) {
  std::vector<double> row(h->G * 5);
  cudaMemcpy(row.data(), h->d_lastStats, h->G * 5 * sizeof(double),
             cudaMemcpyDeviceToHost);
  if (stats)
    for (size_t g = 0; g < h->G; g++) {
      stats[g].maxDisp = row[5 * g + 0];
      stats[g].speed = row[5 * g + 1];
      stats[g].meanAttractive = row[5 * g + 2];
      stats[g].meanRepulsive = row[5 * g + 3];
      stats[g].meanGravity = row[5 * g + 4];
    }
  return row[0];
}

}  // namespace

// ---- shared helpers declared in internal.cuh -----------------------------

int gviz_check(gvizCudaForce *h, cudaError_t e) {
  return e == cudaSuccess ? GVIZ_CUDA_OK : set_err(h, GVIZ_CUDA_ERR_CUDA);
}

void prof_mark(gvizCudaForce *h, const char *name) {
  if (!h->profiling || h->nProf >= 63) return;
  h->profName[h->nProf] = name;
  cudaEventRecord(h->profEv[h->nProf + 1], h->stream);
  h->nProf++;
}

// ---- judge of the learned walk ------------------------------------------

__global__ void k_judge_gather(const double2 *__restrict__ rep, const uint32_t *__restrict__ idx,
                               uint32_t n, double2 *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = rep[idx[i]];
}

// The sampled vertices of the checks: `n` distinct ids drawn with a seeded
// splitmix64 (Floyd's method), ascending.
static std::vector<uint32_t> judge_sample(size_t V, size_t n, uint64_t seed) {
  std::vector<uint32_t> out;
  if (n >= V) {
    out.resize(V);
    for (size_t i = 0; i < V; i++) out[i] = (uint32_t)i;
    return out;
  }
  uint64_t st = seed * 0x9e3779b97f4a7c15ULL + 0x7f4a7c159e3779b9ULL;
  auto next = [&st]() {
    uint64_t z = (st += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  };
  std::vector<uint8_t> taken(V, 0);
  for (size_t j = V - n; j < V; j++) {
    const size_t t = (size_t)(next() % (uint64_t)(j + 1));
    const size_t pick = taken[t] ? j : t;
    taken[pick] = 1;
  }
  out.reserve(n);
  for (size_t i = 0; i < V; i++)
    if (taken[i]) out.push_back((uint32_t)i);
  return out;
}

// One force-only evaluation of the current configuration; the sampled
// vertices' repulsion goes to out (device).
static void judge_eval(gvizCudaForce *h, double2 *out) {
  h->forceOnly = true;
  h->repVecOut = h->d_judgeRep;
  enqueue_step(h);
  h->forceOnly = false;
  h->repVecOut = nullptr;
  k_judge_gather<<<(h->judgeN + 255) / 256, 256, 0, h->stream>>>(h->d_judgeRep, h->d_judgeIdx,
                                                                  h->judgeN, out);
}

// The learned walk judged by the plain one on sampled vertices: the
// normalised RMS error of each against exact FP64 repulsion
// (sqrt(sum |F - F_exact|^2 / sum |F_exact|^2) over the sample). When the
// learned error is above judgeSlack times the plain walk's at judgeTheta,
// the learned walk is turned off (farField = 0): the plain walk is its
// fallback. The layout state is not touched.
static int far_judge(gvizCudaForce *h) {
  if (!h->params.farField || !h->d_mlp || h->V == 0) return GVIZ_CUDA_OK;
  const uint32_t n = (uint32_t)std::min<size_t>(h->judgeSamples, h->V);
  if (n != h->judgeN || !h->d_judgeIdx) {
    dfree(h->d_judgeIdx);
    dfree(h->d_judgeExact);
    dfree(h->d_judgeOut);
    h->judgeN = 0;
    int rc = dalloc(h, &h->d_judgeIdx, n) | dalloc(h, &h->d_judgeExact, n) |
             dalloc(h, &h->d_judgeOut, 2 * (size_t)n);
    if (!h->d_judgeRep) rc |= dalloc(h, &h->d_judgeRep, h->V);
    if (rc) return set_err(h, GVIZ_CUDA_ERR_ALLOC);
    const std::vector<uint32_t> idx = judge_sample(h->V, n, h->judgeSeed);
    if (cudaMemcpy(h->d_judgeIdx, idx.data(), n * 4, cudaMemcpyHostToDevice) != cudaSuccess)
      return set_err(h, GVIZ_CUDA_ERR_CUDA);
    h->judgeN = n;
  }
  cudaMemsetAsync(h->d_status, 0, 4, h->stream);
  enqueue_exact_judge(h, h->d_judgeIdx, n, h->d_judgeExact);
  judge_eval(h, h->d_judgeOut);  // the learned walk as configured
  const gvizCudaForceParams saved = h->params;
  const bool savedSide = h->farSide;
  h->params.farField = 0;
  h->params.theta = h->judgeTheta;
  h->farSide = false;
  judge_eval(h, h->d_judgeOut + n);  // the plain walk
  h->params = saved;
  h->farSide = savedSide;
  int rc = sync_and_check(h);
  if (rc) return rc;
  std::vector<double2> ex(n), got(2 * (size_t)n);
  if (cudaMemcpy(ex.data(), h->d_judgeExact, n * 16, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(got.data(), h->d_judgeOut, 2 * (size_t)n * 16, cudaMemcpyDeviceToHost) !=
          cudaSuccess)
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  double den = 0.0, eL = 0.0, eP = 0.0;
  for (uint32_t i = 0; i < n; i++) {
    const double2 e = ex[i], l = got[i], p = got[n + i];
    den += e.x * e.x + e.y * e.y;
    eL += (l.x - e.x) * (l.x - e.x) + (l.y - e.y) * (l.y - e.y);
    eP += (p.x - e.x) * (p.x - e.x) + (p.y - e.y) * (p.y - e.y);
  }
  h->judgeLearned = den > 0.0 ? sqrt(eL / den) : 0.0;
  h->judgePlain = den > 0.0 ? sqrt(eP / den) : 0.0;
  h->judgeChecks++;
  if (!(h->judgeLearned <= h->judgeSlack * h->judgePlain)) {  // NaN falls back too
    h->params.farField = 0;
    h->farSide = false;
    h->judgeFell = 1;
  }
  h->graphDirty = true;  // the checks ran other work on the step's buffers
  return GVIZ_CUDA_OK;
}

// ---- C ABI ---------------------------------------------------------------

extern "C" {

void gvizCudaForceDefaultParams(gvizCudaForceParams *p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->edgeLength = 10.0;        // GVIZ_FORCE_EMBEDDER_EDGE_LENGTH_DEFAULT
  p->theta = 1.0;              // GVIZ_FORCE_EMBEDDER_THETA_DEFAULT
  p->nodesPerCell = 1;         // GVIZ_QUADTREE_NODES_PER_CELL_DEFAULT
  p->barnesHutEnabled = 1;
  p->gravityK = 0.0;
  p->radiusBase = 0.0;
  p->radiusPerDegree = 0.0;
  p->overlapConstant = 100.0;  // GVIZ_FORCE_EMBEDDER_OVERLAP_CONSTANT_DEFAULT
  p->preventOverlap = 0;
  p->precision = GVIZ_CUDA_FP32;
  p->jitterTolerance = 1.0;    // GVIZ_FORCE_EMBEDDER_JITTER_TOLERANCE_DEFAULT
  p->strictReductions = 0;
  p->farField = 0;
  p->farGroupSpread = 1.0;
  p->farCellGroups = 0;
  p->farHubTargets = 0;
  p->farHubTheta = 0.35;
}

int gvizCudaForceCreate(gvizCudaForce **out, const gvizCudaGraphDesc *g) {
  if (!out || !g) return GVIZ_CUDA_ERR_ARG;
  *out = nullptr;
  const size_t V = g->vertexCount;
  const size_t G = g->graphCount ? g->graphCount : 1;
  if (V > 0 && (!g->rowOffsets || (g->rowOffsets[V] > 0 && !g->neighbors)))
    return GVIZ_CUDA_ERR_ARG;
  if (G > 1 && !g->graphOffsets) return GVIZ_CUDA_ERR_ARG;
  if (g->model != GVIZ_CUDA_MODEL_FR && g->model != GVIZ_CUDA_MODEL_LINLOG)
    return GVIZ_CUDA_ERR_ARG;
  if (V >= 0x7fffffffull / 3 || (V && g->rowOffsets[V] >= 0xffffffffull))
    return GVIZ_CUDA_ERR_LIMIT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
    return GVIZ_CUDA_ERR_NO_DEVICE;
  if (g->device < 0 || g->device >= ndev) return GVIZ_CUDA_ERR_ARG;

  gvizCudaForce *h = new (std::nothrow) gvizCudaForce();
  if (!h) return GVIZ_CUDA_ERR_ALLOC;
  h->device = g->device;
  DeviceGuard guard(h->device);
  h->model = g->model;
  h->V = V;
  h->G = G;
  h->E2 = V ? g->rowOffsets[V] : 0;
  gvizCudaForceDefaultParams(&h->params);
  int gb = 0;
  while (G > 1 && (1ull << gb) < G) gb++;
  if (gb & 1) gb++;
  h->gbits = G > 1 ? gb : 0;
  if (h->gbits > 40) {
    delete h;
    return GVIZ_CUDA_ERR_LIMIT;
  }

  // graph offsets, validation, degree, mass, chunks (host)
  std::vector<uint64_t> goff(G + 1);
  if (G == 1) {
    goff[0] = 0;
    goff[1] = V;
  } else {
    for (size_t i = 0; i <= G; i++) goff[i] = g->graphOffsets[i];
  }
  if (goff[0] != 0 || goff[G] != V) {
    delete h;
    return GVIZ_CUDA_ERR_ARG;
  }
  std::vector<uint32_t> gid(G > 1 ? V : 0);
  for (size_t gg = 0; gg < G; gg++) {
    if (goff[gg + 1] < goff[gg]) {
      delete h;
      return GVIZ_CUDA_ERR_ARG;
    }
    if (G > 1)
      for (uint64_t v = goff[gg]; v < goff[gg + 1]; v++) gid[v] = (uint32_t)gg;
  }
  std::vector<uint32_t> row(V + 1), deg(V ? V : 1);
  std::vector<double> mass(V ? V : 1);
  std::vector<float> massF(V ? V : 1);
  for (size_t v = 0; v <= V; v++) row[v] = (uint32_t)(V ? g->rowOffsets[v] : 0);
  for (size_t v = 0; v < V; v++) {
    if (g->rowOffsets[v + 1] < g->rowOffsets[v]) {
      delete h;
      return GVIZ_CUDA_ERR_ARG;
    }
    uint64_t d = g->degree ? g->degree[v] : g->rowOffsets[v + 1] - g->rowOffsets[v];
    deg[v] = (uint32_t)d;
    // gvizForceModel vertexMass, src/embedders/gvizForceModel.c:5-8, 31
    mass[v] = g->model == GVIZ_CUDA_MODEL_FR ? 1.0 : 1.0 + (double)d;
    massF[v] = (float)mass[v];
  }
  for (uint64_t e = 0; e < h->E2; e++) {
    uint32_t u = g->neighbors[e];
    if (u >= V) {
      delete h;
      return GVIZ_CUDA_ERR_ARG;
    }
  }
  if (G > 1) {  // edges must stay inside their graph
    for (size_t v = 0; v < V; v++)
      for (uint64_t e = g->rowOffsets[v]; e < g->rowOffsets[v + 1]; e++)
        if (gid[g->neighbors[e]] != gid[v]) {
          delete h;
          return GVIZ_CUDA_ERR_ARG;
        }
  }
  std::vector<double> mdp(G);
  for (size_t gg = 0; gg < G; gg++) {
    // meanDegreePlusOne, src/embedders/gvizForceEmbedder.c:251-259
    double s = 0.0;
    for (uint64_t v = goff[gg]; v < goff[gg + 1]; v++) s += (double)(deg[v] + 1);
    uint64_t n = goff[gg + 1] - goff[gg];
    mdp[gg] = n ? s / (double)n : 0.0;
  }
  std::vector<uint32_t> cb, ce, cg, gcb(G), gce(G);
  for (size_t gg = 0; gg < G; gg++) {
    gcb[gg] = (uint32_t)cb.size();
    for (uint64_t s = goff[gg]; s < goff[gg + 1]; s += GVIZ_CHUNK) {
      cb.push_back((uint32_t)s);
      ce.push_back((uint32_t)std::min<uint64_t>(s + GVIZ_CHUNK, goff[gg + 1]));
      cg.push_back((uint32_t)gg);
    }
    gce[gg] = (uint32_t)cb.size();
  }
  h->nChunks = (uint32_t)cb.size();
  std::vector<uint32_t> light, heavy, hubV, hubFirst, hcV, hcE0, hcE1;
  for (size_t v = 0; v < V; v++) {
    const uint64_t d = row[v + 1] - row[v];
    if (d <= GVIZ_HEAVY_DEGREE) {
      light.push_back((uint32_t)v);
    } else if (d <= GVIZ_HUB_DEGREE) {
      heavy.push_back((uint32_t)v);
    } else {
      hubV.push_back((uint32_t)v);
      hubFirst.push_back((uint32_t)hcV.size());
      for (uint64_t e = row[v]; e < row[v + 1]; e += GVIZ_HUB_CHUNK) {
        hcV.push_back((uint32_t)v);
        hcE0.push_back((uint32_t)e);
        hcE1.push_back((uint32_t)std::min<uint64_t>(e + GVIZ_HUB_CHUNK, row[v + 1]));
      }
    }
  }
  hubFirst.push_back((uint32_t)hcV.size());
  h->nAttrLight = (uint32_t)light.size();
  h->nAttrHeavy = (uint32_t)heavy.size();
  h->nHubs = (uint32_t)hubV.size();
  h->nHubChunks = (uint32_t)hcV.size();
  h->h_graphOff = (uint64_t *)malloc(sizeof(uint64_t) * (G + 1));
  h->h_meanDegPlusOne = (double *)malloc(sizeof(double) * G);
  memcpy(h->h_graphOff, goff.data(), sizeof(uint64_t) * (G + 1));
  memcpy(h->h_meanDegPlusOne, mdp.data(), sizeof(double) * G);

  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return GVIZ_CUDA_ERR_CUDA;
  }
  h->ownStream = true;
  if (cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->evFork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->evJoin, cudaEventDisableTiming) != cudaSuccess) {
    if (h->side) cudaStreamDestroy(h->side);
    if (h->evFork) cudaEventDestroy(h->evFork);
    h->side = nullptr;
    h->evFork = nullptr;
    h->evJoin = nullptr;  // without them the attraction runs in order
  }
  const size_t Vs = V ? V : 1;
  const size_t C = h->nChunks ? h->nChunks : 1;
  h->maxNodes = 3 * Vs + 64;
  int rc = 0;
  rc |= dalloc(h, &h->d_rowOff, V + 1);
  rc |= dalloc(h, &h->d_cols, h->E2);
  rc |= dalloc(h, &h->d_degree, Vs);
  rc |= dalloc(h, &h->d_mass, Vs);
  rc |= dalloc(h, &h->d_massF, Vs);
  rc |= dalloc(h, &h->d_radius, Vs);
  rc |= dalloc(h, &h->d_radiusF, Vs);
  if (G > 1) rc |= dalloc(h, &h->d_gid, Vs);
  rc |= dalloc(h, &h->d_graphOff, G + 1);
  rc |= dalloc(h, &h->d_meanDegPlusOne, G);
  rc |= dalloc(h, &h->d_chunkBegin, C);
  rc |= dalloc(h, &h->d_chunkEnd, C);
  rc |= dalloc(h, &h->d_chunkGraph, C);
  rc |= dalloc(h, &h->d_gChunkBegin, G);
  rc |= dalloc(h, &h->d_gChunkEnd, G);
  rc |= dalloc(h, &h->d_attrLight, light.size());
  rc |= dalloc(h, &h->d_attrHeavy, heavy.size());
  rc |= dalloc(h, &h->d_hubV, hubV.size());
  rc |= dalloc(h, &h->d_hubFirst, hubFirst.size());
  rc |= dalloc(h, &h->d_hubChunkV, hcV.size());
  rc |= dalloc(h, &h->d_hubChunkE0, hcE0.size());
  rc |= dalloc(h, &h->d_hubChunkE1, hcE1.size());
  rc |= dalloc(h, &h->d_hubPartial, hcV.size());
  rc |= dalloc(h, &h->d_pos, Vs);
  rc |= dalloc(h, &h->d_sf, Vs);
  rc |= dalloc(h, &h->d_sfOld, Vs);
  rc |= dalloc(h, &h->d_disp, Vs);
  rc |= dalloc(h, &h->d_applied, Vs);
  rc |= dalloc(h, &h->d_att, Vs);
  rc |= dalloc(h, &h->d_rep, Vs);
  rc |= dalloc(h, &h->d_swing, Vs);
  rc |= dalloc(h, &h->d_trac, Vs);
  rc |= dalloc(h, &h->d_attF, Vs);
  rc |= dalloc(h, &h->d_attD, Vs);
  rc |= dalloc(h, &h->d_speed, G);
  rc |= dalloc(h, &h->d_eff, G);
  rc |= dalloc(h, &h->d_active, G);
  rc |= dalloc(h, &h->d_anyActive, 1);
  rc |= dalloc(h, &h->d_iter, G);
  rc |= dalloc(h, &h->d_runLeft, G);
  rc |= dalloc(h, &h->d_runEps, G);
  rc |= dalloc(h, &h->d_stats, (size_t)GVIZ_STATS_CAP * G * 5);
  rc |= dalloc(h, &h->d_lastStats, G * 5);
  rc |= dalloc(h, &h->d_chunkStat, C);
  rc |= dalloc(h, &h->d_status, 1);
  rc |= dalloc(h, &h->d_chunkBox, C);
  rc |= dalloc(h, &h->d_roots, G);
  rc |= dalloc(h, &h->d_keyHi, Vs);
  rc |= dalloc(h, &h->d_keyLo, Vs);
  rc |= dalloc(h, &h->d_ck, Vs);
  rc |= dalloc(h, &h->d_ckAlt, Vs);
  rc |= dalloc(h, &h->d_idx, Vs);
  rc |= dalloc(h, &h->d_idxAlt, Vs);
  rc |= dalloc(h, &h->d_sHi, Vs);
  rc |= dalloc(h, &h->d_sLo, Vs);
  rc |= dalloc(h, &h->d_flag, Vs);
  rc |= dalloc(h, &h->d_scan, Vs);
  rc |= dalloc(h, &h->d_deepRuns, 2 * Vs);
  rc |= dalloc(h, &h->d_counts, 8);
  rc |= dalloc(h, &h->d_sortState, sort_state_entries(Vs));
  rc |= dalloc(h, &h->d_scanState, scan_state_entries(2 * Vs + G));
  rc |= dalloc(h, &h->d_bHi, Vs);
  rc |= dalloc(h, &h->d_bLo, Vs);
  rc |= dalloc(h, &h->d_bGid, Vs);
  rc |= dalloc(h, &h->d_bStart, Vs);
  rc |= dalloc(h, &h->d_nLeft, Vs);
  rc |= dalloc(h, &h->d_nRight, Vs);
  rc |= dalloc(h, &h->d_nFirst, Vs);
  rc |= dalloc(h, &h->d_nLast, Vs);
  rc |= dalloc(h, &h->d_nDelta, Vs);
  rc |= dalloc(h, &h->d_nCounter, Vs);
  rc |= dalloc(h, &h->d_upInt, Vs);
  rc |= dalloc(h, &h->d_upLeaf, Vs);
  rc |= dalloc(h, &h->d_nM, Vs);
  rc |= dalloc(h, &h->d_nSX, Vs);
  rc |= dalloc(h, &h->d_nSY, Vs);
  rc |= dalloc(h, &h->d_nCnt, Vs);
  rc |= dalloc(h, &h->d_nT, Vs);
  rc |= dalloc(h, &h->d_nFlag, Vs);
  rc |= dalloc(h, &h->d_bM, Vs);
  rc |= dalloc(h, &h->d_bSX, Vs);
  rc |= dalloc(h, &h->d_bSY, Vs);
  rc |= dalloc(h, &h->d_bCnt, Vs);
  rc |= dalloc(h, &h->d_bT, Vs);
  rc |= dalloc(h, &h->d_rootNode, G);
  rc |= dalloc(h, &h->d_rootT, G);
  rc |= dalloc(h, &h->d_graphBase, G);
  rc |= dalloc(h, &h->d_nodes, h->maxNodes * sizeof(NodeD));
  rc |= dalloc(h, &h->d_kids, h->maxNodes);
  {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    h->exactSplits = exact_splits(V, sms);
    if (h->exactSplits > 1) rc |= dalloc(h, &h->d_exactPartial, (size_t)h->exactSplits * V);
  }
  rc |= dalloc(h, &h->d_leafDepth, Vs);
  rc |= dalloc(h, &h->d_counters, 8);
  rc |= dalloc(h, &h->d_walkQueue, 1);
  // walk tasks: 32 consecutive path-sorted targets of one graph each, cut
  // from every graph's first sorted position, so that a graph's tasks are
  // the same alone and in a forest
  std::vector<uint2> tasks;
  for (size_t gg = 0; gg < G; gg++)
    for (uint64_t s0 = goff[gg]; s0 < goff[gg + 1]; s0 += 32)
      tasks.push_back(make_uint2((uint32_t)s0, (uint32_t)std::min<uint64_t>(32, goff[gg + 1] - s0)));
  h->nWalkTasks = (uint32_t)tasks.size();
  rc |= dalloc(h, &h->d_walkTasks, std::max<size_t>(tasks.size(), 1));
  if (rc) {
    gvizCudaForceDestroy(h);
    return GVIZ_CUDA_ERR_ALLOC;
  }
  bool ok = true;
  auto up = [&](void *dst, const void *src, size_t bytes) {
    if (bytes && cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) ok = false;
  };
  up(h->d_rowOff, row.data(), (V + 1) * 4);
  if (h->E2) up(h->d_cols, g->neighbors, h->E2 * 4);
  up(h->d_degree, deg.data(), V * 4);
  up(h->d_mass, mass.data(), V * 8);
  up(h->d_massF, massF.data(), V * 4);
  if (G > 1) up(h->d_gid, gid.data(), V * 4);
  up(h->d_graphOff, goff.data(), (G + 1) * 8);
  up(h->d_walkTasks, tasks.data(), tasks.size() * sizeof(uint2));
  up(h->d_meanDegPlusOne, mdp.data(), G * 8);
  up(h->d_chunkBegin, cb.data(), cb.size() * 4);
  up(h->d_chunkEnd, ce.data(), ce.size() * 4);
  up(h->d_chunkGraph, cg.data(), cg.size() * 4);
  up(h->d_gChunkBegin, gcb.data(), G * 4);
  up(h->d_gChunkEnd, gce.data(), G * 4);
  up(h->d_attrLight, light.data(), light.size() * 4);
  up(h->d_attrHeavy, heavy.data(), heavy.size() * 4);
  up(h->d_hubV, hubV.data(), hubV.size() * 4);
  up(h->d_hubFirst, hubFirst.data(), hubFirst.size() * 4);
  up(h->d_hubChunkV, hcV.data(), hcV.size() * 4);
  up(h->d_hubChunkE0, hcE0.data(), hcE0.size() * 4);
  up(h->d_hubChunkE1, hcE1.data(), hcE1.size() * 4);
  ok = ok && cudaMemset(h->d_nCounter, 0, Vs * 4) == cudaSuccess;
  ok = ok && cudaMemset(h->d_pos, 0, Vs * 16) == cudaSuccess;
  ok = ok && cudaMemset(h->d_counters, 0, 64) == cudaSuccess;
  if (!ok || upload_dir_table(h) || upload_radius(h)) {
    gvizCudaForceDestroy(h);
    return GVIZ_CUDA_ERR_CUDA;
  }
  tree_set_smem_limits();
  sort_set_smem_limits();
  forces_set_smem_limits();
  for (int i = 0; i < 65; i++) cudaEventCreate(&h->profEv[i]);
  // Init leaves the FA2 state zeroed (src/embedders/gvizForceEmbedder.c:221);
  // Begin sets it up.
  ok = cudaMemset(h->d_speed, 0, G * 8) == cudaSuccess &&
       cudaMemset(h->d_eff, 0, G * 8) == cudaSuccess &&
       cudaMemset(h->d_sf, 0, Vs * 16) == cudaSuccess &&
       cudaMemset(h->d_iter, 0, G * 8) == cudaSuccess &&
       cudaMemset(h->d_lastStats, 0, G * 40) == cudaSuccess;
  if (!ok) {
    gvizCudaForceDestroy(h);
    return GVIZ_CUDA_ERR_CUDA;
  }
  set_all_active(h, ~0ull, -INFINITY);
  *out = h;
  return GVIZ_CUDA_OK;
}

void gvizCudaForceDestroy(gvizCudaForce *h) {
  if (!h) return;
  DeviceGuard guard(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->stepExec) cudaGraphExecDestroy(h->stepExec);
  for (int i = 0; i < 65; i++)
    if (h->profEv[i]) cudaEventDestroy(h->profEv[i]);
  free_all(h);
  mlp_free(h);
  far_side_free(h);
  if (h->upload) {
    cudaStreamSynchronize(h->upload);
    cudaStreamDestroy(h->upload);
  }
  if (h->evUp) cudaEventDestroy(h->evUp);
  for (int c = 0; c < GVIZ_HOST_PIECES; c++)
    if (h->evDown[c]) cudaEventDestroy(h->evDown[c]);
  if (h->side) {
    cudaStreamSynchronize(h->side);
    cudaStreamDestroy(h->side);
  }
  if (h->evFork) cudaEventDestroy(h->evFork);
  if (h->evJoin) cudaEventDestroy(h->evJoin);
  cudaFree(h->d_farHubs);
  cudaFree(h->d_farHubOut);
  if (h->ownStream && h->stream) cudaStreamDestroy(h->stream);
  free(h->h_graphOff);
  free(h->h_meanDegPlusOne);
  delete h;
}

// The `count` heaviest vertices (model mass; ties to the lower id), in id
// order, as the learned walk's hub targets.
static int select_hubs(gvizCudaForce *h, uint32_t count) {
  if (h->stream) cudaStreamSynchronize(h->stream);
  h->graphDirty = true;  // the captured step holds the buffers freed here
  cudaFree(h->d_farHubs);
  cudaFree(h->d_farHubOut);
  h->d_farHubs = nullptr;
  h->d_farHubOut = nullptr;
  h->nFarHubs = 0;
  if (count == 0) return GVIZ_CUDA_OK;
  std::vector<double> mass(h->V);
  if (cudaMemcpy(mass.data(), h->d_mass, h->V * sizeof(double), cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return GVIZ_CUDA_ERR_CUDA;
  std::vector<uint32_t> ids(h->V);
  for (size_t i = 0; i < h->V; i++) ids[i] = (uint32_t)i;
  auto heavier = [&](uint32_t a, uint32_t b) {
    return mass[a] > mass[b] || (mass[a] == mass[b] && a < b);
  };
  std::nth_element(ids.begin(), ids.begin() + (count - 1), ids.end(), heavier);
  std::sort(ids.begin(), ids.begin() + count);
  // the ids, then the walk's hub counter
  if (cudaMalloc(&h->d_farHubs, (count + 1) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&h->d_farHubOut, count * sizeof(double2)) != cudaSuccess) {
    cudaFree(h->d_farHubs);
    h->d_farHubs = nullptr;
    return GVIZ_CUDA_ERR_ALLOC;
  }
  if (cudaMemcpy(h->d_farHubs, ids.data(), count * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return GVIZ_CUDA_ERR_CUDA;
  h->nFarHubs = count;
  return GVIZ_CUDA_OK;
}

int gvizCudaForceSetParams(gvizCudaForce *h, const gvizCudaForceParams *p) {
  if (!h || !p) return GVIZ_CUDA_ERR_ARG;
  if (p->nodesPerCell < 1 || p->nodesPerCell > GVIZ_MAX_NODES_PER_CELL)
    return set_err(h, GVIZ_CUDA_ERR_LIMIT);
  if (!(p->theta > 0.0) || !(p->edgeLength > 0.0) ||
      (p->precision != GVIZ_CUDA_FP32 && p->precision != GVIZ_CUDA_FP64))
    return set_err(h, GVIZ_CUDA_ERR_ARG);
  // the learned correction lives in the FP32 walk and needs a model
  if (p->farField && (!h->d_mlp || p->precision != GVIZ_CUDA_FP32 || !p->barnesHutEnabled))
    return set_err(h, GVIZ_CUDA_ERR_ARG);
  if (!(p->farGroupSpread >= 0.0 && p->farGroupSpread <= 1.0) ||
      (p->farCellGroups != 0 && p->farCellGroups != 1) || p->farHubTargets < 0 ||
      (p->farHubTargets > 0 && !(p->farHubTheta > 0.0 && p->farHubTheta < INFINITY)))
    return set_err(h, GVIZ_CUDA_ERR_ARG);
  DeviceGuard guard(h->device);
  const uint32_t hubs = (uint32_t)std::min<size_t>((size_t)p->farHubTargets, h->V);
  if (hubs != h->nFarHubs) {
    const int rc = select_hubs(h, hubs);
    if (rc) return set_err(h, rc);
  }
  const bool radiusChanged = p->preventOverlap != h->params.preventOverlap ||
                             p->radiusBase != h->params.radiusBase ||
                             p->radiusPerDegree != h->params.radiusPerDegree;
  h->params = *p;
  h->farSide = p->farField != 0;
  h->graphDirty = true;
  if (radiusChanged) return upload_radius(h);
  return GVIZ_CUDA_OK;
}

int gvizCudaForceGetParams(const gvizCudaForce *h, gvizCudaForceParams *p) {
  if (!h || !p) return GVIZ_CUDA_ERR_ARG;
  *p = h->params;
  return GVIZ_CUDA_OK;
}

int gvizCudaForceSetPositions(gvizCudaForce *h, const double *xy) {
  if (!h || (!xy && h->V)) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  if (!h->V) return GVIZ_CUDA_OK;
  if (cudaMemcpyAsync(h->d_pos, xy, h->V * 16, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  return GVIZ_CUDA_OK;
}

int gvizCudaForceGetPositions(gvizCudaForce *h, double *xy) {
  if (!h || (!xy && h->V)) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  if (!h->V) return GVIZ_CUDA_OK;
  if (cudaMemcpyAsync(xy, h->d_pos, h->V * 16, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  return GVIZ_CUDA_OK;
}

int gvizCudaForceBegin(gvizCudaForce *h) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  std::vector<double> one(h->G, 1.0);
  bool ok = cudaMemcpy(h->d_speed, one.data(), h->G * 8, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(h->d_eff, one.data(), h->G * 8, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemset(h->d_sf, 0, (h->V ? h->V : 1) * 16) == cudaSuccess;
  ok = ok && cudaMemset(h->d_disp, 0, (h->V ? h->V : 1) * 16) == cudaSuccess;
  ok = ok && cudaMemset(h->d_iter, 0, h->G * 8) == cudaSuccess;
  ok = ok && cudaMemset(h->d_lastStats, 0, h->G * 40) == cudaSuccess;
  if (!ok) return set_err(h, GVIZ_CUDA_ERR_CUDA);
  set_all_active(h, ~0ull, -INFINITY);
  h->begun = true;
  h->hostIteration = 0;
  return GVIZ_CUDA_OK;
}

int gvizCudaForceSetFa2State(gvizCudaForce *h, const double *sf,
                             const double *speed, const double *eff) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  bool ok = true;
  if (sf && h->V) ok = cudaMemcpy(h->d_sf, sf, h->V * 16, cudaMemcpyHostToDevice) == cudaSuccess;
  if (speed) ok = ok && cudaMemcpy(h->d_speed, speed, h->G * 8, cudaMemcpyHostToDevice) == cudaSuccess;
  if (eff) ok = ok && cudaMemcpy(h->d_eff, eff, h->G * 8, cudaMemcpyHostToDevice) == cudaSuccess;
  return ok ? GVIZ_CUDA_OK : set_err(h, GVIZ_CUDA_ERR_CUDA);
}

int gvizCudaForceGetFa2State(gvizCudaForce *h, double *sf, double *speed,
                             double *eff) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return set_err(h, GVIZ_CUDA_ERR_CUDA);
  bool ok = true;
  if (sf && h->V) ok = cudaMemcpy(sf, h->d_sf, h->V * 16, cudaMemcpyDeviceToHost) == cudaSuccess;
  if (speed) ok = ok && cudaMemcpy(speed, h->d_speed, h->G * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
  if (eff) ok = ok && cudaMemcpy(eff, h->d_eff, h->G * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
  return ok ? GVIZ_CUDA_OK : set_err(h, GVIZ_CUDA_ERR_CUDA);
}

double gvizCudaForceStep(gvizCudaForce *h, gvizCudaStepStats *stats) {
  if (!h) return (double)GVIZ_CUDA_ERR_ARG;
  if (!h->begun) return (double)set_err(h, GVIZ_CUDA_ERR_NOT_BEGUN);
  DeviceGuard guard(h->device);
  if (h->V == 0) {
    // the reference still appends stats for an empty graph
    if (stats)
      for (size_t g = 0; g < h->G; g++) {
        memset(&stats[g], 0, sizeof(stats[g]));
        stats[g].speed = 1.0;
      }
    return 0.0;
  }
  int rc = launch_steps(h, 1);
  if (rc) return (double)rc;
  rc = sync_and_check(h);
  h->hostIteration++;
  double md = fill_stats(h, stats);
  return rc ? (double)rc : md;
}

double gvizCudaForceStepHost(gvizCudaForce *h, double *xy,
                             gvizCudaStepStats *stats) {
  if (!h || (!xy && h->V)) return (double)GVIZ_CUDA_ERR_ARG;
  if (!h->begun) return (double)set_err(h, GVIZ_CUDA_ERR_NOT_BEGUN);
  DeviceGuard guard(h->device);
  if (h->V == 0) return gvizCudaForceStep(h, stats);
  if (cudaMemcpyAsync(h->d_pos, xy, h->V * 16, cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
    return (double)set_err(h, GVIZ_CUDA_ERR_CUDA);
  int rc = launch_steps(h, 1);
  if (rc) return (double)rc;
  if (cudaMemcpyAsync(xy, h->d_pos, h->V * 16, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
    return (double)set_err(h, GVIZ_CUDA_ERR_CUDA);
  rc = sync_and_check(h);
  h->hostIteration++;
  double md = fill_stats(h, stats);
  return rc ? (double)rc : md;
}

// Streams and events of gvizCudaForceRunHost, made once per handle.
static int host_pipeline(gvizCudaForce *h) {
  if (h->upload) return GVIZ_CUDA_OK;
  cudaStream_t up = nullptr;
  if (cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking) != cudaSuccess)
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  bool ok = cudaEventCreateWithFlags(&h->evUp, cudaEventDisableTiming) == cudaSuccess;
  for (int c = 0; ok && c < GVIZ_HOST_PIECES; c++)
    ok = cudaEventCreateWithFlags(&h->evDown[c], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    if (h->evUp) cudaEventDestroy(h->evUp);
    h->evUp = nullptr;
    for (int c = 0; c < GVIZ_HOST_PIECES; c++) {
      if (h->evDown[c]) cudaEventDestroy(h->evDown[c]);
      h->evDown[c] = nullptr;
    }
    cudaStreamDestroy(up);
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  }
  h->upload = up;
  return GVIZ_CUDA_OK;
}

double gvizCudaForceRunHost(gvizCudaForce *h, double *xy, uint32_t steps,
                            gvizCudaStepStats *stats) {
  if (!h || (!xy && h->V)) return (double)GVIZ_CUDA_ERR_ARG;
  if (!h->begun) return (double)set_err(h, GVIZ_CUDA_ERR_NOT_BEGUN);
  DeviceGuard guard(h->device);
  if (steps == 0) {
    int rc = sync_and_check(h);
    return rc ? (double)rc : fill_stats(h, stats);
  }
  if (h->V == 0) {
    double md = 0.0;
    for (uint32_t k = 0; k < steps; k++) {
      md = gvizCudaForceStep(h, stats);
      if (md < 0) return md;
    }
    return md;
  }
  int rc = host_pipeline(h);
  if (rc) return (double)rc;
  const size_t doubles = 2 * h->V;
  const size_t piece = (doubles + GVIZ_HOST_PIECES - 1) / GVIZ_HOST_PIECES;
  bool ok = cudaMemcpyAsync(h->d_pos, xy, doubles * 8, cudaMemcpyHostToDevice, h->stream) ==
            cudaSuccess;
  double *dpos = reinterpret_cast<double *>(h->d_pos);
  for (uint32_t k = 0; ok && k < steps; k++) {
    rc = launch_steps(h, 1);
    if (rc) return (double)rc;
    const bool again = k + 1 < steps;
    for (int c = 0; ok && c < GVIZ_HOST_PIECES; c++) {
      const size_t off = (size_t)c * piece;
      if (off >= doubles) break;
      const size_t n = std::min(piece, doubles - off);
      ok = cudaMemcpyAsync(xy + off, dpos + off, n * 8, cudaMemcpyDeviceToHost, h->stream) ==
           cudaSuccess;
      if (ok && again) {  // the next step's upload of this piece, once it is back
        ok = cudaEventRecord(h->evDown[c], h->stream) == cudaSuccess &&
             cudaStreamWaitEvent(h->upload, h->evDown[c], 0) == cudaSuccess &&
             cudaMemcpyAsync(dpos + off, xy + off, n * 8, cudaMemcpyHostToDevice,
                             h->upload) == cudaSuccess;
      }
    }
    if (ok && again)
      ok = cudaEventRecord(h->evUp, h->upload) == cudaSuccess &&
           cudaStreamWaitEvent(h->stream, h->evUp, 0) == cudaSuccess;
  }
  if (!ok) return (double)set_err(h, GVIZ_CUDA_ERR_CUDA);
  rc = sync_and_check(h);
  h->hostIteration += steps;
  double md = fill_stats(h, stats);
  return rc ? (double)rc : md;
}

int gvizCudaForceEnqueueSteps(gvizCudaForce *h, uint32_t n) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  if (!h->begun) return set_err(h, GVIZ_CUDA_ERR_NOT_BEGUN);
  DeviceGuard guard(h->device);
  int rc = launch_steps(h, n);
  if (!rc) h->hostIteration += n;
  return rc;
}

int gvizCudaForceSynchronize(gvizCudaForce *h) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  return sync_and_check(h);
}

int gvizCudaForceRun(gvizCudaForce *h, size_t maxIters, double epsilon,
                     uint64_t *rounds) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  if (!h->begun) return set_err(h, GVIZ_CUDA_ERR_NOT_BEGUN);
  DeviceGuard guard(h->device);
  std::vector<uint64_t> it0(h->G), it1(h->G);
  cudaMemcpy(it0.data(), h->d_iter, h->G * 8, cudaMemcpyDeviceToHost);
  if (maxIters > 0 && h->V > 0) {
    set_all_active(h, maxIters, epsilon);
    size_t launched = 0;
    while (launched < maxIters) {
      uint32_t n = (uint32_t)std::min<size_t>(kRunBatch, maxIters - launched);
      int rc = launch_steps(h, n);
      if (rc) return rc;
      launched += n;
      uint32_t any = 0;
      if (cudaMemcpyAsync(&any, h->d_anyActive, 4, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
        return set_err(h, GVIZ_CUDA_ERR_CUDA);
      int sc = sync_and_check(h);
      if (sc) return sc;
      if (any == 0) break;
    }
    set_all_active(h, ~0ull, -INFINITY);
  }
  cudaMemcpy(it1.data(), h->d_iter, h->G * 8, cudaMemcpyDeviceToHost);
  if (rounds)
    for (size_t g = 0; g < h->G; g++) rounds[g] = it1[g] - it0[g];
  h->hostIteration += it1[0] - it0[0];
  return GVIZ_CUDA_OK;
}

int64_t gvizCudaForceStatHistory(gvizCudaForce *h, uint32_t graph, double *out,
                                 size_t cap) {
  if (!h || graph >= h->G) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  cudaStreamSynchronize(h->stream);
  uint64_t it = 0;
  cudaMemcpy(&it, h->d_iter + graph, 8, cudaMemcpyDeviceToHost);
  const uint64_t kept = std::min<uint64_t>(it, GVIZ_STATS_CAP);
  const uint64_t first = it - kept;
  uint64_t w = 0;
  for (uint64_t s = first; s < it && w < cap; s++, w++) {
    const size_t rowIdx = (size_t)(s % GVIZ_STATS_CAP);
    if (out)
      cudaMemcpy(out + 5 * w, h->d_stats + (rowIdx * h->G + graph) * 5,
                 5 * sizeof(double), cudaMemcpyDeviceToHost);
  }
  return (int64_t)kept;
}

int gvizCudaForceGetForces(gvizCudaForce *h, double *disp, double *sf,
                           double *att, double *rep, double *swing,
                           double *trac, double *applied) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return set_err(h, GVIZ_CUDA_ERR_CUDA);
  const size_t V = h->V;
  if (!V) return GVIZ_CUDA_OK;
  bool ok = true;
  auto dn = [&](void *dst, const void *src, size_t bytes) {
    if (dst && cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) ok = false;
  };
  dn(disp, h->d_disp, V * 16);
  dn(sf, h->d_sf, V * 16);
  dn(att, h->d_att, V * 8);
  dn(rep, h->d_rep, V * 8);
  dn(swing, h->d_swing, V * 8);
  dn(trac, h->d_trac, V * 8);
  dn(applied, h->d_applied, V * 16);
  return ok ? GVIZ_CUDA_OK : set_err(h, GVIZ_CUDA_ERR_CUDA);
}

static uint64_t mask_hi(int d) {
  if (d <= 0) return 0;
  if (d >= 32) return ~0ull;
  return ~0ull << (64 - 2 * d);
}
static uint64_t mask_lo(int d) {
  if (d <= 32) return 0;
  if (d >= 64) return ~0ull;
  return ~0ull << (128 - 2 * d);
}

int gvizCudaForceTreeLeaves(gvizCudaForce *h, int32_t *leafDepth,
                            uint64_t *pathHi, uint64_t *pathLo,
                            uint64_t *nodeCount) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  const size_t V = h->V;
  if (V == 0) {
    if (nodeCount) *nodeCount = 0;
    return GVIZ_CUDA_OK;
  }
  cudaMemsetAsync(h->d_status, 0, 4, h->stream);
  enqueue_tree_build(h);
  enqueue_tree_export(h, (int32_t *)h->d_leafDepth);
  int rc = sync_and_check(h);
  if (rc) return rc;
  std::vector<int32_t> depth(V);
  std::vector<uint64_t> hi(V), lo(V);
  std::vector<uint32_t> idx(V);
  uint32_t counts[8];
  bool ok = cudaMemcpy(depth.data(), h->d_leafDepth, V * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
  ok = ok && cudaMemcpy(hi.data(), h->d_sHi, V * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
  ok = ok && cudaMemcpy(lo.data(), h->d_sLo, V * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
  ok = ok && cudaMemcpy(idx.data(), h->d_idx, V * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
  ok = ok && cudaMemcpy(counts, h->d_counts, 32, cudaMemcpyDeviceToHost) == cudaSuccess;
  if (!ok) return set_err(h, GVIZ_CUDA_ERR_CUDA);
  for (size_t s = 0; s < V; s++) {
    const uint32_t v = idx[s];
    const int d = depth[v];
    if (leafDepth) leafDepth[v] = d;
    if (pathHi) pathHi[v] = hi[s] & mask_hi(d);
    if (pathLo) pathLo[v] = lo[s] & mask_lo(d);
  }
  if (nodeCount) *nodeCount = counts[3];
  return GVIZ_CUDA_OK;
}

int64_t gvizCudaForceTreeNodes(gvizCudaForce *h, size_t cap, int32_t *depth,
                               uint64_t *pathHi, uint64_t *pathLo,
                               double *mass, double *comX, double *comY,
                               uint64_t *count) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  if (h->V == 0) return 0;
  const size_t M = h->maxNodes;
  int32_t *dd = nullptr;
  uint64_t *dh = nullptr, *dl = nullptr, *dc = nullptr;
  double *dm = nullptr, *dx = nullptr, *dy = nullptr;
  int rc = 0;
  rc |= dalloc(h, &dd, M);
  rc |= dalloc(h, &dh, M);
  rc |= dalloc(h, &dl, M);
  rc |= dalloc(h, &dc, M);
  rc |= dalloc(h, &dm, M);
  rc |= dalloc(h, &dx, M);
  rc |= dalloc(h, &dy, M);
  int64_t w = 0;
  if (!rc) {
    cudaMemsetAsync(dd, 0xff, M * 4, h->stream);
    cudaMemsetAsync(h->d_status, 0, 4, h->stream);
    enqueue_tree_build(h);
    enqueue_cell_dump(h, dd, dh, dl, dm, dx, dy, dc);
    rc = sync_and_check(h);
    if (!rc) {
      std::vector<int32_t> D(M);
      std::vector<uint64_t> H(M), L(M), Cn(M);
      std::vector<double> Ms(M), X(M), Y(M);
      cudaMemcpy(D.data(), dd, M * 4, cudaMemcpyDeviceToHost);
      cudaMemcpy(H.data(), dh, M * 8, cudaMemcpyDeviceToHost);
      cudaMemcpy(L.data(), dl, M * 8, cudaMemcpyDeviceToHost);
      cudaMemcpy(Cn.data(), dc, M * 8, cudaMemcpyDeviceToHost);
      cudaMemcpy(Ms.data(), dm, M * 8, cudaMemcpyDeviceToHost);
      cudaMemcpy(X.data(), dx, M * 8, cudaMemcpyDeviceToHost);
      cudaMemcpy(Y.data(), dy, M * 8, cudaMemcpyDeviceToHost);
      for (size_t i = 0; i < M; i++) {
        if (D[i] < 0) continue;
        if ((size_t)w < cap) {
          if (depth) depth[w] = D[i];
          if (pathHi) pathHi[w] = H[i];
          if (pathLo) pathLo[w] = L[i];
          if (mass) mass[w] = Ms[i];
          if (comX) comX[w] = X[i];
          if (comY) comY[w] = Y[i];
          if (count) count[w] = Cn[i];
        }
        w++;
      }
    }
  }
  dfree(dd);
  dfree(dh);
  dfree(dl);
  dfree(dc);
  dfree(dm);
  dfree(dx);
  dfree(dy);
  return rc ? (int64_t)rc : w;
}

int gvizCudaForceExactRepulsion(gvizCudaForce *h, const uint32_t *targets,
                                size_t n, double *out) {
  if (!h || (n && (!targets || !out))) return GVIZ_CUDA_ERR_ARG;
  if (n == 0) return GVIZ_CUDA_OK;
  for (size_t i = 0; i < n; i++)
    if (targets[i] >= h->V) return set_err(h, GVIZ_CUDA_ERR_ARG);
  DeviceGuard guard(h->device);
  uint32_t *dt = nullptr;
  double2 *dout = nullptr;
  int rc = dalloc(h, &dt, n) | dalloc(h, &dout, n);
  if (!rc) {
    cudaMemcpy(dt, targets, n * 4, cudaMemcpyHostToDevice);
    enqueue_exact_judge(h, dt, n, dout);
    rc = sync_and_check(h);
    if (!rc && cudaMemcpy(out, dout, n * 16, cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = set_err(h, GVIZ_CUDA_ERR_CUDA);
  }
  dfree(dt);
  dfree(dout);
  return rc;
}

int gvizCudaForceRepulsion(gvizCudaForce *h, double *out) {
  if (!h || (!out && h->V)) return GVIZ_CUDA_ERR_ARG;
  if (h->V == 0) return GVIZ_CUDA_OK;
  DeviceGuard guard(h->device);
  double2 *dv = nullptr;
  int rc = dalloc(h, &dv, h->V);
  if (!rc) {
    h->forceOnly = true;
    h->repVecOut = dv;
    cudaMemsetAsync(h->d_status, 0, 4, h->stream);
    enqueue_step(h);
    h->forceOnly = false;
    h->repVecOut = nullptr;
    rc = sync_and_check(h);
    if (!rc && cudaMemcpy(out, dv, h->V * 16, cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = set_err(h, GVIZ_CUDA_ERR_CUDA);
  }
  dfree(dv);
  return rc;
}

// One instrumented force evaluation: c = {pair interactions, warp node
// visits, learned-correction shared rows, lane rows, lane rows by cause:
// too few accepting targets, spread too wide, centroid fails the opening
// test, warp iterations that accepted a cell}.
static int count_walk(gvizCudaForce *h, uint64_t c[8]) {
  const gvizCudaForceParams saved = h->params;
  h->params.precision = GVIZ_CUDA_FP32;
  h->forceOnly = true;
  cudaMemsetAsync(h->d_counters, 0, 64, h->stream);
  cudaMemsetAsync(h->d_status, 0, 4, h->stream);
  enqueue_tree_build(h);
  enqueue_attraction_f32(h);
  enqueue_walk_f32(h, h->d_counters);
  h->forceOnly = false;
  h->params = saved;
  int rc = sync_and_check(h);
  if (cudaMemcpy(c, h->d_counters, 64, cudaMemcpyDeviceToHost) != cudaSuccess && !rc)
    rc = set_err(h, GVIZ_CUDA_ERR_CUDA);
  return rc;
}

int gvizCudaForceCountInteractions(gvizCudaForce *h, uint64_t *interactions,
                                   uint64_t *warpNodeVisits) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  if (h->V == 0 || !h->params.barnesHutEnabled) {
    const uint64_t n = h->V;
    if (interactions) *interactions = h->params.barnesHutEnabled ? 0 : n * (n ? n - 1 : 0);
    if (warpNodeVisits) *warpNodeVisits = 0;
    return GVIZ_CUDA_OK;
  }
  uint64_t c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int rc = count_walk(h, c);
  if (interactions) *interactions = c[0];
  if (warpNodeVisits) *warpNodeVisits = c[1];
  return rc;
}

int gvizCudaForceCountFarRows(gvizCudaForce *h, uint64_t *groupRows, uint64_t *laneRows,
                              uint64_t *laneRowCause) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  uint64_t c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int rc = GVIZ_CUDA_OK;
  if (h->V > 0 && h->params.barnesHutEnabled && h->params.farField) rc = count_walk(h, c);
  if (groupRows) *groupRows = c[2];
  if (laneRows) *laneRows = c[3];
  if (laneRowCause) memcpy(laneRowCause, c + 4, 3 * sizeof(uint64_t));
  return rc;
}

int gvizCudaForceProfileStep(gvizCudaForce *h, size_t cap, const char **names,
                             double *ms) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  if (!h->begun) return set_err(h, GVIZ_CUDA_ERR_NOT_BEGUN);
  DeviceGuard guard(h->device);
  if (h->V == 0) return 0;
  h->profiling = true;
  h->nProf = 0;
  cudaEventRecord(h->profEv[0], h->stream);
  enqueue_step(h);
  h->profiling = false;
  int rc = sync_and_check(h);
  h->hostIteration++;
  if (rc) return rc;
  int n = h->nProf;
  for (int i = 0; i < n && (size_t)i < cap; i++) {
    float t = 0.f;
    cudaEventElapsedTime(&t, h->profEv[i], h->profEv[i + 1]);
    if (names) names[i] = h->profName[i];
    if (ms) ms[i] = t;
  }
  return n;
}

int gvizCudaForceTimeSteps(gvizCudaForce *h, uint32_t n, float *ms) {
  if (!h || !ms) return GVIZ_CUDA_ERR_ARG;
  if (!h->begun) return set_err(h, GVIZ_CUDA_ERR_NOT_BEGUN);
  DeviceGuard guard(h->device);
  *ms = 0.f;
  if (h->V == 0 || n == 0) return GVIZ_CUDA_OK;
  int rc = ensure_graph(h);
  if (rc) return rc;
  cudaEventRecord(h->profEv[0], h->stream);
  rc = launch_steps(h, n);
  if (rc) return rc;
  cudaEventRecord(h->profEv[1], h->stream);
  rc = sync_and_check(h);
  h->hostIteration += n;
  if (rc) return rc;
  cudaEventElapsedTime(ms, h->profEv[0], h->profEv[1]);
  return GVIZ_CUDA_OK;
}

int gvizCudaForceStepKernelCount(gvizCudaForce *h) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  if (h->V == 0) return 0;
  DeviceGuard guard(h->device);
  int rc = ensure_graph(h);
  return rc ? rc : h->kernelsPerStep;
}

int gvizCudaForceLastError(const gvizCudaForce *h) {
  return h ? h->lastError : GVIZ_CUDA_ERR_ARG;
}

const char *gvizCudaErrorString(int code) {
  switch (code) {
    case GVIZ_CUDA_OK: return "ok";
    case GVIZ_CUDA_ERR_ALLOC: return "allocation failed";
    case GVIZ_CUDA_ERR_DIMENSION: return "only 2-D layouts are supported";
    case GVIZ_CUDA_ERR_ARG: return "invalid argument";
    case GVIZ_CUDA_ERR_CUDA: return "CUDA runtime error";
    case GVIZ_CUDA_ERR_NOT_BEGUN: return "Begin has not been called";
    case GVIZ_CUDA_ERR_NONFINITE: return "a vertex position is NaN or infinite";
    case GVIZ_CUDA_ERR_DEEP_RUN: return "more than 4096 distinct points share one depth-32 quadtree cell";
    case GVIZ_CUDA_ERR_NO_DEVICE: return "no usable CUDA device";
    case GVIZ_CUDA_ERR_LIMIT: return "size beyond a supported limit";
    default: return "unknown error";
  }
}

int gvizCudaForceSetStream(gvizCudaForce *h, void *stream) {
  if (!h || !stream) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  cudaStreamSynchronize(h->stream);
  if (h->ownStream) cudaStreamDestroy(h->stream);
  h->stream = (cudaStream_t)stream;
  h->ownStream = false;
  h->graphDirty = true;
  return GVIZ_CUDA_OK;
}


// ---- lossless checkpoint ---------------------------------------------------
//
// gviz saves an embedding as text with six decimals and no FA2 speed state
// (src/embedders/gvizEmbeddedGraph.c:428-448), so a run cannot be resumed
// exactly. The binary checkpoint below holds everything a step reads from
// the previous one: positions, structForce (the next step's old force),
// global speed and efficiency, per-graph iteration counters and the stat
// history ring, all as raw little-endian bytes, closed by an FNV-1a 64
// checksum of everything before it. Layout (version 1):
//   "GVZCKPT1" | u32 version | u32 name bytes | u64 V | u64 G | i32 model |
//   i32 dim (2) | u32 params bytes | u32 begun | name | params |
//   u64 graphOffsets[G+1] | f64 positions[2V] | f64 structForce[2V] |
//   f64 speed[G] | f64 efficiency[G] | u64 iteration[G] | u64 host iteration |
//   u64 ring rows R | f64 stats[R][G][5] | f64 lastStats[G][5] | u64 checksum

namespace {

constexpr char kCkptMagic[8] = {'G', 'V', 'Z', 'C', 'K', 'P', 'T', '1'};
constexpr uint32_t kCkptVersion = 1;

struct CkptHeader {
  char magic[8];
  uint32_t version, nameBytes;
  uint64_t V, G;
  int32_t model, dim;
  uint32_t paramsBytes, begun;
};

struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void *p, size_t n) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < n; i++) {
      h ^= b[i];
      h *= 1099511628211ull;
    }
  }
};

struct CkptWriter {
  FILE *f;
  Fnv sum;
  bool ok = true;
  void put(const void *p, size_t n) {
    if (!ok || n == 0) return;
    sum.add(p, n);
    ok = fwrite(p, 1, n, f) == n;
  }
};

struct CkptReader {
  FILE *f;
  Fnv sum;
  bool ok = true;
  void get(void *p, size_t n) {
    if (!ok || n == 0) return;
    ok = fread(p, 1, n, f) == n;
    if (ok) sum.add(p, n);
  }
};

}  // namespace

int gvizCudaForceSaveCheckpoint(gvizCudaForce *h, const char *name, const char *filename) {
  if (!h || !filename) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return set_err(h, GVIZ_CUDA_ERR_CUDA);
  const size_t V = h->V, G = h->G;
  std::vector<double> pos(2 * V), sf(2 * V), speed(G), eff(G), last(5 * G);
  std::vector<uint64_t> iter(G);
  bool ok = true;
  if (V) {
    ok = cudaMemcpy(pos.data(), h->d_pos, V * 16, cudaMemcpyDeviceToHost) == cudaSuccess;
    ok = ok && cudaMemcpy(sf.data(), h->d_sf, V * 16, cudaMemcpyDeviceToHost) == cudaSuccess;
  }
  ok = ok && cudaMemcpy(speed.data(), h->d_speed, G * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
  ok = ok && cudaMemcpy(eff.data(), h->d_eff, G * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
  ok = ok && cudaMemcpy(iter.data(), h->d_iter, G * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
  ok = ok && cudaMemcpy(last.data(), h->d_lastStats, G * 40, cudaMemcpyDeviceToHost) == cudaSuccess;
  uint64_t maxIt = 0;
  for (uint64_t it : iter) maxIt = std::max(maxIt, it);
  const uint64_t rows = std::min<uint64_t>(maxIt, GVIZ_STATS_CAP);
  std::vector<double> ring(rows * G * 5);
  if (rows)
    ok = ok && cudaMemcpy(ring.data(), h->d_stats, ring.size() * 8, cudaMemcpyDeviceToHost) ==
                   cudaSuccess;
  if (!ok) return set_err(h, GVIZ_CUDA_ERR_CUDA);
  FILE *f = fopen(filename, "wb");
  if (!f) return set_err(h, GVIZ_CUDA_ERR_ARG);
  CkptWriter w{f};
  CkptHeader hd;
  memcpy(hd.magic, kCkptMagic, 8);
  hd.version = kCkptVersion;
  hd.nameBytes = name ? (uint32_t)strlen(name) : 0u;
  hd.V = V;
  hd.G = G;
  hd.model = h->model;
  hd.dim = 2;
  hd.paramsBytes = sizeof(gvizCudaForceParams);
  hd.begun = h->begun ? 1u : 0u;
  w.put(&hd, sizeof(hd));
  w.put(name, hd.nameBytes);
  w.put(&h->params, sizeof(gvizCudaForceParams));
  w.put(h->h_graphOff, (G + 1) * 8);
  w.put(pos.data(), pos.size() * 8);
  w.put(sf.data(), sf.size() * 8);
  w.put(speed.data(), G * 8);
  w.put(eff.data(), G * 8);
  w.put(iter.data(), G * 8);
  w.put(&h->hostIteration, 8);
  w.put(&rows, 8);
  w.put(ring.data(), ring.size() * 8);
  w.put(last.data(), last.size() * 8);
  const uint64_t sum = w.sum.h;
  ok = w.ok && fwrite(&sum, 8, 1, f) == 1;
  ok = (fclose(f) == 0) && ok;
  return ok ? GVIZ_CUDA_OK : set_err(h, GVIZ_CUDA_ERR_ARG);
}

int gvizCudaForceLoadCheckpoint(gvizCudaForce *h, const char *filename, int restoreParams,
                                char *nameOut, size_t nameCap) {
  if (!h || !filename) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  FILE *f = fopen(filename, "rb");
  if (!f) return set_err(h, GVIZ_CUDA_ERR_ARG);
  CkptReader r{f};
  CkptHeader hd;
  r.get(&hd, sizeof(hd));
  // the file must be a version-1 checkpoint of this very graph (or forest)
  bool ok = r.ok && memcmp(hd.magic, kCkptMagic, 8) == 0 && hd.version == kCkptVersion &&
            hd.V == h->V && hd.G == h->G && hd.model == h->model && hd.dim == 2 &&
            hd.paramsBytes == sizeof(gvizCudaForceParams) && hd.nameBytes < (1u << 20);
  const size_t V = h->V, G = h->G;
  std::string name(ok ? hd.nameBytes : 0, '\0');
  gvizCudaForceParams params;
  std::vector<uint64_t> goff(G + 1), iter(G);
  std::vector<double> pos(2 * V), sf(2 * V), speed(G), eff(G), last(5 * G);
  uint64_t hostIt = 0, rows = 0;
  if (ok) {
    r.get(&name[0], hd.nameBytes);
    r.get(&params, sizeof(params));
    r.get(goff.data(), (G + 1) * 8);
    ok = r.ok && memcmp(goff.data(), h->h_graphOff, (G + 1) * 8) == 0;
  }
  if (ok) {
    r.get(pos.data(), pos.size() * 8);
    r.get(sf.data(), sf.size() * 8);
    r.get(speed.data(), G * 8);
    r.get(eff.data(), G * 8);
    r.get(iter.data(), G * 8);
    r.get(&hostIt, 8);
    r.get(&rows, 8);
    ok = r.ok && rows <= GVIZ_STATS_CAP;
  }
  std::vector<double> ring(ok ? rows * G * 5 : 0);
  uint64_t stored = 0;
  if (ok) {
    r.get(ring.data(), ring.size() * 8);
    r.get(last.data(), last.size() * 8);
    const uint64_t sum = r.sum.h;
    ok = r.ok && fread(&stored, 8, 1, f) == 1 && stored == sum && fgetc(f) == EOF;
  }
  fclose(f);
  if (!ok) return set_err(h, GVIZ_CUDA_ERR_ARG);  // not this graph's, or damaged
  for (size_t i = 0; i < 2 * V; i++)
    if (!std::isfinite(pos[i])) return set_err(h, GVIZ_CUDA_ERR_NONFINITE);
  if (restoreParams) {
    const int rc = gvizCudaForceSetParams(h, &params);
    if (rc) return rc;
  }
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return set_err(h, GVIZ_CUDA_ERR_CUDA);
  bool cok = true;
  if (V) {
    cok = cudaMemcpy(h->d_pos, pos.data(), V * 16, cudaMemcpyHostToDevice) == cudaSuccess;
    cok = cok && cudaMemcpy(h->d_sf, sf.data(), V * 16, cudaMemcpyHostToDevice) == cudaSuccess;
    cok = cok && cudaMemset(h->d_disp, 0, V * 16) == cudaSuccess;
  }
  cok = cok && cudaMemcpy(h->d_speed, speed.data(), G * 8, cudaMemcpyHostToDevice) == cudaSuccess;
  cok = cok && cudaMemcpy(h->d_eff, eff.data(), G * 8, cudaMemcpyHostToDevice) == cudaSuccess;
  cok = cok && cudaMemcpy(h->d_iter, iter.data(), G * 8, cudaMemcpyHostToDevice) == cudaSuccess;
  cok = cok && cudaMemcpy(h->d_lastStats, last.data(), G * 40, cudaMemcpyHostToDevice) == cudaSuccess;
  if (rows)
    cok = cok && cudaMemcpy(h->d_stats, ring.data(), ring.size() * 8, cudaMemcpyHostToDevice) ==
                     cudaSuccess;
  if (!cok) return set_err(h, GVIZ_CUDA_ERR_CUDA);
  set_all_active(h, ~0ull, -INFINITY);
  h->begun = hd.begun != 0;
  h->hostIteration = hostIt;
  if (nameOut && nameCap) {
    const size_t n = std::min(nameCap - 1, name.size());
    memcpy(nameOut, name.data(), n);
    nameOut[n] = '\0';
  }
  return GVIZ_CUDA_OK;
}

int gvizCudaForceSaveEmbeddingText(gvizCudaForce *h, const char *name, const char *filename) {
  if (!h || !filename) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return set_err(h, GVIZ_CUDA_ERR_CUDA);
  std::vector<double> pos(2 * h->V);
  if (h->V && cudaMemcpy(pos.data(), h->d_pos, h->V * 16, cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_err(h, GVIZ_CUDA_ERR_CUDA);
  FILE *f = fopen(filename, "w");
  if (!f) return set_err(h, GVIZ_CUDA_ERR_ARG);
  // gviz's layout (src/embedders/gvizEmbeddedGraph.c:428-448): name line,
  // "count dim", one row per vertex; 17 significant digits instead of %f,
  // so gvizEmbeddedGraphLoadEmbedding's %lf reads every bit back
  bool ok = fprintf(f, "%s\n%zu %d\n", name ? name : "", h->V, 2) > 0;
  for (size_t i = 0; ok && i < h->V; i++)
    ok = fprintf(f, "%.17g %.17g \n", pos[2 * i], pos[2 * i + 1]) > 0;
  ok = (fclose(f) == 0) && ok;
  return ok ? GVIZ_CUDA_OK : set_err(h, GVIZ_CUDA_ERR_ARG);
}


// ---- walk launch autotuning ------------------------------------------------

int gvizCudaForceAutotune(gvizCudaForce *h, uint32_t *threadsOut, int32_t *persistentOut,
                          float *walkMsOut) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  if (h->V == 0 || !h->params.barnesHutEnabled || h->params.farField ||
      h->params.precision != GVIZ_CUDA_FP32)
    return GVIZ_CUDA_OK;  // only the FP32 plain walk has launch choices
  static const uint32_t kCandidates[] = {64, 128, 256, 512};
  const gvizCudaForceParams saved = h->params;
  h->forceOnly = true;
  cudaMemsetAsync(h->d_status, 0, 4, h->stream);
  enqueue_tree_build(h);
  enqueue_attraction_f32(h);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = INFINITY;
  uint32_t bestThreads = kWalkDefaultThreads;
  bool bestPersistent = false;
  uint32_t bestResident = 0, bestCap = 0;
  // stack entries per warp: a smaller stack takes less shared memory, so
  // more warps are resident, and walks more subtrees in place; a cap set by
  // the caller is kept
  static const uint32_t kCaps[] = {128, 256, 512};
  const int nCaps = h->walkStackCap ? 1 : 3;
  for (int ci = 0; ci < nCaps; ci++)
  for (int persistent = 0; persistent < 2; persistent++) {
    for (uint32_t t : kCandidates) {
      h->walkTunedCap = h->walkStackCap ? 0u : kCaps[ci];
      h->walkThreads = t;
      h->walkPersistent = persistent != 0;
      h->walkResident = persistent ? walk_resident_blocks(h, t) : 0;
      if (persistent && !h->walkResident) continue;
      enqueue_walk_f32(h, nullptr);  // warm-up; forces-only launches repeat cleanly
      float ms = INFINITY;
      for (int r = 0; r < 3; r++) {
        cudaEventRecord(e0, h->stream);
        enqueue_walk_f32(h, nullptr);
        cudaEventRecord(e1, h->stream);
        float m = 0.f;
        if (cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&m, e0, e1) == cudaSuccess)
          ms = std::min(ms, m);
      }
      if (ms < best) {
        best = ms;
        bestThreads = t;
        bestPersistent = persistent != 0;
        bestResident = h->walkResident;
        bestCap = h->walkTunedCap;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->forceOnly = false;
  h->params = saved;
  h->walkThreads = bestThreads;
  h->walkPersistent = bestPersistent;
  h->walkResident = bestResident;
  h->walkTunedCap = bestCap;
  h->graphDirty = true;
  const int rc = sync_and_check(h);
  if (threadsOut) *threadsOut = bestThreads;
  if (persistentOut) *persistentOut = bestPersistent ? 1 : 0;
  if (walkMsOut) *walkMsOut = best;
  return rc;
}


int gvizCudaForceSetFarJudge(gvizCudaForce *h, uint32_t every, uint32_t samples,
                             double plainTheta, double slack, uint64_t seed) {
  if (!h || samples == 0 || !(plainTheta > 0.0 && plainTheta < INFINITY) ||
      !(slack > 0.0 && slack < INFINITY))
    return GVIZ_CUDA_ERR_ARG;
  if (samples != h->judgeSamples || seed != h->judgeSeed) h->judgeN = 0;  // new sample
  h->judgeEvery = every;
  h->judgeSamples = samples;
  h->judgeTheta = plainTheta;
  h->judgeSlack = slack;
  h->judgeSeed = seed;
  h->judgeNextAt = h->stepsLaunched;  // the next learned step is checked first
  return GVIZ_CUDA_OK;
}

int gvizCudaForceJudgeFarField(gvizCudaForce *h, double *learnedErr, double *plainErr,
                               int32_t *fellBack) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  if (!h->begun) return set_err(h, GVIZ_CUDA_ERR_NOT_BEGUN);
  DeviceGuard guard(h->device);
  const int32_t was = h->params.farField;
  h->judgeLearned = h->judgePlain = 0.0;
  const int rc = far_judge(h);
  if (learnedErr) *learnedErr = h->judgeLearned;
  if (plainErr) *plainErr = h->judgePlain;
  if (fellBack) *fellBack = (was && !h->params.farField) ? 1 : 0;
  return rc;
}

int gvizCudaForceFarJudgeStatus(const gvizCudaForce *h, uint64_t *checks, double *learnedErr,
                                double *plainErr, int32_t *fellBack) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  if (checks) *checks = h->judgeChecks;
  if (learnedErr) *learnedErr = h->judgeLearned;
  if (plainErr) *plainErr = h->judgePlain;
  if (fellBack) *fellBack = h->judgeFell;
  return GVIZ_CUDA_OK;
}

int gvizCudaForceSetWalkStackCap(gvizCudaForce *h, uint32_t entries) {
  if (!h || (entries != 0 && (entries < 32 || entries > 512))) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  h->walkStackCap = entries;
  // the persistent grid of the plain walk follows its shared memory
  if (h->walkPersistent) {
    const uint32_t resident = walk_resident_blocks(h, h->walkThreads ? h->walkThreads
                                                                      : kWalkDefaultThreads);
    if (!resident) return set_err(h, GVIZ_CUDA_ERR_CUDA);
    h->walkResident = resident;
  }
  h->graphDirty = true;
  return GVIZ_CUDA_OK;
}

int gvizCudaForceSetWalkShape(gvizCudaForce *h, uint32_t threads, int32_t persistent) {
  if (!h || threads < 32 || threads > 512 || threads % 32 != 0) return GVIZ_CUDA_ERR_ARG;
  DeviceGuard guard(h->device);
  const uint32_t resident = persistent ? walk_resident_blocks(h, threads) : 0;
  if (persistent && !resident) return set_err(h, GVIZ_CUDA_ERR_CUDA);
  h->walkThreads = threads;
  h->walkPersistent = persistent != 0;
  h->walkResident = resident;
  h->graphDirty = true;
  return GVIZ_CUDA_OK;
}

int gvizCudaForceGetWalkShape(const gvizCudaForce *h, uint32_t *threads, int32_t *persistent,
                              uint32_t *stackEntries) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  if (threads) *threads = h->walkThreads ? h->walkThreads : kWalkDefaultThreads;
  if (persistent) *persistent = (h->walkPersistent && h->walkResident) ? 1 : 0;
  if (stackEntries) *stackEntries = plain_cap(h);
  return GVIZ_CUDA_OK;
}

}  // extern "C"
