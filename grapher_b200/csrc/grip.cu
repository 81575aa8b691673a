// grip.cu -- the force phase of gviz's GRIP embedder on the device: one
// refinement round (gvizGRIPEmbedderRefineRound,
// src/embedders/gvizGRIPEmbedder.c:1289-1334) over the active vertices of
// the current layer, given the layer's filtration order and each active
// vertex's k-nearest list (graph distance), which the host builds as GRIP
// does (MIS filtration, placement and the k-nearest search stay on the host).
//
// FP64, compiled without fused multiply-add, every expression in the
// reference's operation order: the per-vertex forces, heat and step are
// bit-identical to the reference's. The sums over the layer (mean
// displacement, centroid, angular momentum, inertia, round statistics) run
// in one block: each thread sums a contiguous chunk in order and thread 0
// adds the chunk sums in order, so they are deterministic; with
// strictReductions one thread sums everything in the reference's serial
// order and the round is bit-identical to the reference's. 2-D only.
#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "gvizcuda.h"

namespace {

// src/embedders/gvizGRIPEmbedder.c:31, 45-46 and
// src/embedders/gvizForceDirected.c:4, include/embedders/gvizForceDirected.h:6
constexpr double kEdge = 10.0;       // GVIZ_EDGE_LENGTH
constexpr double kR = 0.15;          // gvizGRIPr
constexpr double kS = 3;             // gvizGRIPs
constexpr double kFrScale = 0.05;    // FR_SCALE_FACTOR
constexpr double kEps = 1e-7;        // gvizNumericEpsilon
constexpr int kThreads = 256;
constexpr int kSumThreads = 1024;  // room of the partial kernels' staging
constexpr int kPartThreads = 256;
constexpr uint32_t kMaxParts = 592;  // 4 blocks per SM

struct GripArgs {
  const uint64_t *row;
  const uint32_t *col;
  const uint32_t *active;   // the layer in filtration order (sums, move)
  const uint32_t *work;     // the layer in label order (force kernel)
  const uint64_t *knnOff;   // list t (of work[t]) has knnOff[t+1] - knnOff[t] entries
  const uint64_t *warpBase; // lists of warp w start at warpBase[w]
  const uint32_t *knnV, *knnD;  // entry e of list 32w + l at warpBase[w] + 32e + l
  double *part;             // per-block partial sums of the ordered reductions
  double2 *pos, *disp, *oldDisp;
  double *heat, *oldCos, *lastF, *nrm;
  uint8_t *calc;
  double *red;  // [0,1] mean disp, [2,3] centroid, [4] omega, [5] rotate, [6..9] stats
  uint32_t n, layer, parts;  // parts: blocks of the partial-sum kernels
};

constexpr int kBatch = 8;

// gvizVecAccKKForce (include/core/gvizVec.h:138-186) at L = dist * 10
__device__ __forceinline__ void kk_term(double2 p, double2 q, uint32_t dist, double &fx,
                                        double &fy) {
  const double L = (double)dist * kEdge;
  if (L < 1e-9) return;
  const double dx = q.x - p.x, dy = q.y - p.y;
  const double s = sqrt(dx * dx + dy * dy) / L - 1.0;
  fx += s * dx;
  fy += s * dy;
}

// gvizVecAccGRIPFRAttForce (include/core/gvizVec.h:115-180), frScale 0.05
__device__ __forceinline__ void grip_att_term(double2 p, double2 q, double &fx, double &fy) {
  const double dx = p.x - q.x, dy = p.y - q.y;
  const double d2 = dx * dx + dy * dy;
  if (d2 < 1e-18) return;
  const double s = kFrScale * (kEdge * kEdge) / d2;
  fx += s * dx;
  fy += s * dy;
}

// Spring forces (calculateSpringForces :892-934; the ops of
// include/core/gvizVec.h:138-316 via src/embedders/gvizForceDirected.c:6-20),
// then the heat update (:1071-1103 with updateLocalTemp :870-889) and the
// heat-scaled step.
__global__ __launch_bounds__(kThreads) void k_grip_pass1(GripArgs a) {
  const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= a.n) return;
  const uint32_t v = a.work[i];
  const double2 prev = a.disp[v];
  a.oldDisp[v] = prev;
  const double2 p = a.pos[v];
  double fx = 0.0, fy = 0.0;
  // this thread's list, stored warp-interleaved so that the lanes' loads of
  // entry e are coalesced
  const uint32_t len = (uint32_t)(a.knnOff[i + 1] - a.knnOff[i]);
  const uint64_t k0 = a.warpBase[i >> 5] + (i & 31u);
  const uint64_t k1 = k0 + 32ull * len;
  // the list is walked in batches of kBatch entries: all their loads are
  // issued first (the gathers are what bounds this kernel), then the terms
  // are added in list order, as the reference adds them
  if (a.layer > 0) {
    uint64_t e = k0;
    for (; e + 32ull * (kBatch - 1) < k1; e += 32ull * kBatch) {  // KK springs
      uint32_t dist[kBatch];
      double2 q[kBatch];
#pragma unroll
      for (int j = 0; j < kBatch; j++) dist[j] = a.knnD[e + 32ull * j];
#pragma unroll
      for (int j = 0; j < kBatch; j++) q[j] = a.pos[a.knnV[e + 32ull * j]];
#pragma unroll
      for (int j = 0; j < kBatch; j++) kk_term(p, q[j], dist[j], fx, fy);
    }
    for (; e < k1; e += 32) kk_term(p, a.pos[a.knnV[e]], a.knnD[e], fx, fy);
  } else {
    const double lenSq = kEdge * kEdge;
    for (uint64_t j = a.row[v]; j < a.row[v + 1]; j++) {  // along edges
      const double2 q = a.pos[a.col[j]];
      const double dx = q.x - p.x, dy = q.y - p.y;
      const double d2 = dx * dx + dy * dy;
      if (d2 < 1e-18) continue;
      const double s = d2 / lenSq;
      fx += s * dx;
      fy += s * dy;
    }
    uint64_t e = k0;
    for (; e + 32ull * (kBatch - 1) < k1; e += 32ull * kBatch) {  // from the k nearest
      double2 q[kBatch];
#pragma unroll
      for (int j = 0; j < kBatch; j++) q[j] = a.pos[a.knnV[e + 32ull * j]];
#pragma unroll
      for (int j = 0; j < kBatch; j++) grip_att_term(p, q[j], fx, fy);
    }
    for (; e < k1; e += 32) grip_att_term(p, a.pos[a.knnV[e]], fx, fy);
  }
  double heat = a.heat[v], oc = a.oldCos[v];
  if (!a.calc[v]) {
    a.calc[v] = 1;
    heat = kEdge / 6.0;
  } else {
    const double nrm = sqrt(fx * fx + fy * fy);
    const double oldNrm = sqrt(prev.x * prev.x + prev.y * prev.y);
    if (!(fabs(nrm) < kEps || fabs(oldNrm) < kEps)) {
      const double c = (fx * prev.x + fy * prev.y) / (nrm * oldNrm);
      if (c > 0 && oc > 0)
        heat *= (1 + c * kR * kS);
      else
        heat *= (1 + c * kR);
      oc = c;
    }
  }
  heat = fmin(heat, kEdge * 10);
  heat = fmax(heat, kEdge * 1e-4);
  const double nrm = sqrt(fx * fx + fy * fy);
  a.lastF[v] = nrm;
  if (nrm > kEps) {
    const double s = heat / nrm;
    fx *= s;
    fy *= s;
  }
  a.disp[v] = make_double2(fx, fy);
  a.heat[v] = heat;
  a.oldCos[v] = oc;
}

// Ordered sums over the layer in two launches. Partial: block b takes the
// contiguous range of items [b*B, (b+1)*B); each thread sums a contiguous
// chunk of it in order and thread 0 adds the chunk sums in order. Final:
// one thread adds the block partials in order. Deterministic; with one block
// of one thread (strict reductions) the whole sum runs in the reference's
// serial order.
template <int K>
__device__ __forceinline__ void block_partial(double (&acc)[K], double *out,
                                              double (*tmp)[K]) {
  for (int k = 0; k < K; k++) tmp[threadIdx.x][k] = acc[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < K; k++) acc[k] = tmp[0][k];
    for (unsigned t = 1; t < blockDim.x; t++)
      for (int k = 0; k < K; k++) acc[k] += tmp[t][k];
    for (int k = 0; k < K; k++) out[blockIdx.x * K + k] = acc[k];
  }
}

__device__ __forceinline__ void item_range(uint32_t n, uint32_t &b, uint32_t &e) {
  const uint32_t per = (n + gridDim.x - 1) / gridDim.x;
  const uint32_t lo = blockIdx.x * per, hi = min(lo + per, n);
  const uint32_t c = (per + blockDim.x - 1) / blockDim.x;
  b = min(lo + threadIdx.x * c, hi);
  e = min(b + c, hi);
}

// sums of the displacements and the positions (removeNetTranslation
// :1106-1121, the centroid of removeNetRotation :1192-1203)
__global__ __launch_bounds__(kSumThreads) void k_grip_part1(GripArgs a) {
  __shared__ double tmp[kSumThreads][4];
  uint32_t b, e;
  item_range(a.n, b, e);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t i = b; i < e; i++) {
    const uint32_t v = a.active[i];
    const double2 d = a.disp[v], p = a.pos[v];
    acc[0] += 1.0 * d.x;
    acc[1] += 1.0 * d.y;
    acc[2] += p.x;
    acc[3] += p.y;
  }
  block_partial<4>(acc, a.part, tmp);
}

// the block partials, loaded by the whole block into shared memory so that
// one thread can add them in order without waiting on each load
__device__ __forceinline__ const double *stage_parts(const GripArgs &a, double *sp) {
  for (uint32_t j = threadIdx.x; j < a.parts * 4; j += blockDim.x) sp[j] = a.part[j];
  __syncthreads();
  return sp;
}

__global__ __launch_bounds__(kPartThreads) void k_grip_final1(GripArgs a) {
  __shared__ double sp[kMaxParts * 4];
  const double *part = stage_parts(a, sp);
  if (threadIdx.x) return;
  double acc[4];
  for (int k = 0; k < 4; k++) acc[k] = part[k];
  for (uint32_t b = 1; b < a.parts; b++)
    for (int k = 0; k < 4; k++) acc[k] += part[b * 4 + k];
  const double inv = 1.0 / (double)a.n;
  a.red[0] = acc[0] * inv;
  a.red[1] = acc[1] * inv;
  a.red[2] = acc[2] / (double)a.n;
  a.red[3] = acc[3] / (double)a.n;
}

// angular momentum of the translated displacements and the polar moment of
// inertia about the centroid; omega = L / I (:1204-1252, dim 2)
__global__ __launch_bounds__(kSumThreads) void k_grip_part2(GripArgs a) {
  __shared__ double tmp[kSumThreads][2];
  uint32_t b, e;
  item_range(a.n, b, e);
  const double mx = a.red[0], my = a.red[1], cx = a.red[2], cy = a.red[3];
  double acc[2] = {0.0, 0.0};
  for (uint32_t i = b; i < e; i++) {
    const uint32_t v = a.active[i];
    const double2 p = a.pos[v];
    double2 d = a.disp[v];
    d.x += -1.0 * mx;
    d.y += -1.0 * my;
    const double rx = p.x - cx, ry = p.y - cy;
    acc[0] += rx * d.y - ry * d.x;
    acc[1] += rx * rx + ry * ry;
  }
  block_partial<2>(acc, a.part, tmp);
}

__global__ __launch_bounds__(kPartThreads) void k_grip_final2(GripArgs a) {
  __shared__ double sp[kMaxParts * 4];
  const double *part = stage_parts(a, sp);
  if (threadIdx.x) return;
  double L = part[0], I = part[1];
  for (uint32_t b = 1; b < a.parts; b++) {
    L += part[b * 2];
    I += part[b * 2 + 1];
  }
  const bool rotate = a.n >= 3 && !(fabs(I) < kEps);
  a.red[4] = rotate ? L / I : 0.0;
  a.red[5] = rotate ? 1.0 : 0.0;
}

// remove the translation and the rotation, move (gvizEmbeddedGraphAdd-
// VPosition, src/embedders/gvizEmbeddedGraph.c:400-404)
__global__ __launch_bounds__(kThreads) void k_grip_apply(GripArgs a) {
  const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= a.n) return;
  const uint32_t v = a.active[i];
  const double2 p = a.pos[v];
  double2 d = a.disp[v];
  d.x += -1.0 * a.red[0];
  d.y += -1.0 * a.red[1];
  if (a.red[5] != 0.0) {
    const double w = a.red[4];
    const double rx = p.x - a.red[2], ry = p.y - a.red[3];
    d.x -= 0.0 * 0.0 - w * ry;
    d.y -= w * rx - 0.0 * 0.0;
  }
  a.disp[v] = d;
  a.nrm[i] = sqrt(d.x * d.x + d.y * d.y);
  a.pos[v] = make_double2(p.x + 1.0 * d.x, p.y + 1.0 * d.y);
}

// round statistics (:1302-1331): max and sums of |disp|, heat, force
__global__ __launch_bounds__(kSumThreads) void k_grip_part3(GripArgs a) {
  __shared__ double tmp[kSumThreads][4];
  uint32_t b, e;
  item_range(a.n, b, e);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};  // max, sum disp, sum heat, sum force
  for (uint32_t i = b; i < e; i++) {
    const uint32_t v = a.active[i];
    const double nrm = a.nrm[i];
    if (nrm > acc[0]) acc[0] = nrm;
    acc[1] += nrm;
    acc[2] += a.heat[v];
    acc[3] += a.lastF[v];
  }
  tmp[threadIdx.x][0] = acc[0];
  __syncthreads();
  double mx = acc[0];
  if (threadIdx.x == 0)
    for (unsigned t = 1; t < blockDim.x; t++) mx = fmax(mx, tmp[t][0]);
  __syncthreads();
  block_partial<4>(acc, a.part, tmp);
  if (threadIdx.x == 0) a.part[blockIdx.x * 4] = mx;
}

__global__ __launch_bounds__(kPartThreads) void k_grip_final3(GripArgs a) {
  __shared__ double sp[kMaxParts * 4];
  const double *part = stage_parts(a, sp);
  if (threadIdx.x) return;
  double mx = part[0], acc[3] = {part[1], part[2], part[3]};
  for (uint32_t b = 1; b < a.parts; b++) {
    mx = fmax(mx, part[b * 4]);
    for (int k = 0; k < 3; k++) acc[k] += part[b * 4 + 1 + k];
  }
  a.red[6] = mx;
  a.red[7] = a.n ? acc[0] / a.n : 0.0;
  a.red[8] = a.n ? acc[1] / a.n : 0.0;
  a.red[9] = a.n ? acc[2] / a.n : 0.0;
}

// clearDecorators (:936-951) for the vertices of the new layer
__global__ __launch_bounds__(kThreads) void k_grip_clear(GripArgs a) {
  const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= a.n) return;
  const uint32_t v = a.active[i];
  a.heat[v] = 0.0;
  a.oldCos[v] = 0.0;
  a.disp[v] = make_double2(0.0, 0.0);
  a.oldDisp[v] = make_double2(0.0, 0.0);
}

inline uint32_t grid_for(size_t n) { return (uint32_t)((n + kThreads - 1) / kThreads); }

}  // namespace

struct gvizCudaGrip {
  int device = 0;
  cudaStream_t stream = nullptr;
  size_t V = 0, E2 = 0;
  int strict = 0;
  uint64_t *d_row = nullptr;
  uint32_t *d_col = nullptr;
  double2 *d_pos = nullptr, *d_disp = nullptr, *d_old = nullptr;
  double *d_heat = nullptr, *d_oldCos = nullptr, *d_lastF = nullptr, *d_nrm = nullptr;
  double *d_red = nullptr;
  uint8_t *d_calc = nullptr;
  uint32_t *d_active = nullptr, *d_knnV = nullptr, *d_knnD = nullptr;
  uint64_t *d_knnOff = nullptr, *d_warpBase = nullptr;
  double *d_part = nullptr;  // kMaxParts x 4 partial sums
  uint32_t *d_work = nullptr;
  size_t n = 0, knnCap = 0, layer = 0;
  bool hasLayer = false;
  // Vertices are relabelled in breadth-first order inside the handle (old
  // id perm[n] is label n), so that graph-near vertices, whose k-nearest
  // lists overlap, sit near each other in memory and in the force kernel's
  // warps. The API keeps the caller's ids.
  std::vector<uint32_t> perm, inv;
};

namespace {

template <typename T>
int galloc(T **p, size_t count) {
  return cudaMalloc(reinterpret_cast<void **>(p), (count ? count : 1) * sizeof(T)) == cudaSuccess
             ? GVIZ_CUDA_OK
             : GVIZ_CUDA_ERR_ALLOC;
}

struct GripGuard {
  int prev = 0;
  explicit GripGuard(int dev) {
    cudaGetDevice(&prev);
    cudaSetDevice(dev);
  }
  ~GripGuard() { cudaSetDevice(prev); }
};

GripArgs grip_args(gvizCudaGrip *h) {
  GripArgs a;
  a.row = h->d_row;
  a.col = h->d_col;
  a.active = h->d_active;
  a.work = h->d_work;
  a.knnOff = h->d_knnOff;
  a.warpBase = h->d_warpBase;
  a.part = h->d_part;
  a.knnV = h->d_knnV;
  a.knnD = h->d_knnD;
  a.pos = h->d_pos;
  a.disp = h->d_disp;
  a.oldDisp = h->d_old;
  a.heat = h->d_heat;
  a.oldCos = h->d_oldCos;
  a.lastF = h->d_lastF;
  a.nrm = h->d_nrm;
  a.calc = h->d_calc;
  a.red = h->d_red;
  a.n = (uint32_t)h->n;
  a.layer = (uint32_t)h->layer;
  const uint32_t want = (uint32_t)((h->n + 1023) / 1024);
  a.parts = h->strict ? 1u : (want < 1 ? 1u : (want > kMaxParts ? kMaxParts : want));
  return a;
}

void grip_free(gvizCudaGrip *h) {
  cudaFree(h->d_row);
  cudaFree(h->d_col);
  cudaFree(h->d_pos);
  cudaFree(h->d_disp);
  cudaFree(h->d_old);
  cudaFree(h->d_heat);
  cudaFree(h->d_oldCos);
  cudaFree(h->d_lastF);
  cudaFree(h->d_nrm);
  cudaFree(h->d_red);
  cudaFree(h->d_calc);
  cudaFree(h->d_active);
  cudaFree(h->d_knnOff);
  cudaFree(h->d_warpBase);
  cudaFree(h->d_part);
  cudaFree(h->d_work);
  cudaFree(h->d_knnV);
  cudaFree(h->d_knnD);
}

}  // namespace

extern "C" {

int gvizCudaGripCreate(gvizCudaGrip **out, size_t vertexCount, const uint64_t *rowOffsets,
                       const uint32_t *neighbors, int32_t device) {
  if (!out || (vertexCount && !rowOffsets)) return GVIZ_CUDA_ERR_ARG;
  *out = nullptr;
  if (vertexCount >= 0xffffffffull) return GVIZ_CUDA_ERR_LIMIT;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return GVIZ_CUDA_ERR_NO_DEVICE;
  if (device < 0 || device >= count) return GVIZ_CUDA_ERR_ARG;
  const size_t E2 = vertexCount ? rowOffsets[vertexCount] : 0;
  if (E2 && !neighbors) return GVIZ_CUDA_ERR_ARG;
  for (size_t e = 0; e < E2; e++)
    if (neighbors[e] >= vertexCount) return GVIZ_CUDA_ERR_ARG;
  GripGuard guard(device);
  gvizCudaGrip *h = new gvizCudaGrip;
  h->device = device;
  h->V = vertexCount;
  h->E2 = E2;
  const size_t V = vertexCount;
  int rc = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess
               ? GVIZ_CUDA_OK
               : GVIZ_CUDA_ERR_CUDA;
  if (!rc) rc |= galloc(&h->d_row, V + 1);
  if (!rc) rc |= galloc(&h->d_col, E2);
  if (!rc) rc |= galloc(&h->d_pos, V);
  if (!rc) rc |= galloc(&h->d_disp, V);
  if (!rc) rc |= galloc(&h->d_old, V);
  if (!rc) rc |= galloc(&h->d_heat, V);
  if (!rc) rc |= galloc(&h->d_oldCos, V);
  if (!rc) rc |= galloc(&h->d_lastF, V);
  if (!rc) rc |= galloc(&h->d_nrm, V);
  if (!rc) rc |= galloc(&h->d_red, 16);
  if (!rc) rc |= galloc(&h->d_calc, V);
  if (!rc) rc |= galloc(&h->d_active, V);
  if (!rc) rc |= galloc(&h->d_knnOff, V + 1);
  if (!rc) rc |= galloc(&h->d_warpBase, V / 32 + 2);
  if (!rc) rc |= galloc(&h->d_part, (size_t)kMaxParts * 4);
  if (!rc) rc |= galloc(&h->d_work, V);
  if (rc) {
    grip_free(h);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return rc;
  }
  // breadth-first labels: from the highest-degree vertex, then from every
  // vertex not reached yet, in id order
  h->perm.reserve(V);
  h->inv.assign(V, 0);
  std::vector<uint8_t> seen(V, 0);
  size_t hub = 0;
  for (size_t v = 1; v < V; v++)
    if (rowOffsets[v + 1] - rowOffsets[v] > rowOffsets[hub + 1] - rowOffsets[hub]) hub = v;
  for (size_t k = 0; k <= V; k++) {
    const size_t s0 = k == 0 ? hub : k - 1;
    if (s0 >= V || seen[s0]) continue;
    seen[s0] = 1;
    size_t head = h->perm.size();
    h->perm.push_back((uint32_t)s0);
    for (; head < h->perm.size(); head++) {
      const uint32_t u = h->perm[head];
      for (uint64_t j = rowOffsets[u]; j < rowOffsets[u + 1]; j++) {
        const uint32_t w = neighbors[j];
        if (!seen[w]) {
          seen[w] = 1;
          h->perm.push_back(w);
        }
      }
    }
  }
  for (size_t n = 0; n < V; n++) h->inv[h->perm[n]] = (uint32_t)n;
  // the CSR in labels, each row keeping the caller's neighbour order
  std::vector<uint64_t> row2(V + 1, 0);
  std::vector<uint32_t> col2(E2);
  for (size_t n = 0; n < V; n++) {
    const uint32_t o = h->perm[n];
    row2[n + 1] = row2[n] + (rowOffsets[o + 1] - rowOffsets[o]);
    for (uint64_t j = rowOffsets[o]; j < rowOffsets[o + 1]; j++)
      col2[row2[n] + (j - rowOffsets[o])] = h->inv[neighbors[j]];
  }
  if (V) {
    cudaMemcpyAsync(h->d_row, row2.data(), (V + 1) * 8, cudaMemcpyHostToDevice, h->stream);
    if (E2) cudaMemcpyAsync(h->d_col, col2.data(), E2 * 4, cudaMemcpyHostToDevice, h->stream);
    cudaMemsetAsync(h->d_pos, 0, V * 16, h->stream);
    cudaMemsetAsync(h->d_disp, 0, V * 16, h->stream);
    cudaMemsetAsync(h->d_old, 0, V * 16, h->stream);
    cudaMemsetAsync(h->d_heat, 0, V * 8, h->stream);
    cudaMemsetAsync(h->d_oldCos, 0, V * 8, h->stream);
    cudaMemsetAsync(h->d_lastF, 0, V * 8, h->stream);
    cudaMemsetAsync(h->d_calc, 0, V, h->stream);
  }
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
    grip_free(h);
    cudaStreamDestroy(h->stream);
    delete h;
    return GVIZ_CUDA_ERR_CUDA;
  }
  *out = h;
  return GVIZ_CUDA_OK;
}

void gvizCudaGripDestroy(gvizCudaGrip *h) {
  if (!h) return;
  GripGuard guard(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  grip_free(h);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int gvizCudaGripSetStrictReductions(gvizCudaGrip *h, int32_t strict) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  h->strict = strict != 0;
  return GVIZ_CUDA_OK;
}

int gvizCudaGripSetPositions(gvizCudaGrip *h, const double *xy) {
  if (!h || (h->V && !xy)) return GVIZ_CUDA_ERR_ARG;
  GripGuard guard(h->device);
  if (!h->V) return GVIZ_CUDA_OK;
  std::vector<double> tmp(2 * h->V);
  for (size_t n = 0; n < h->V; n++) {
    tmp[2 * n] = xy[2 * (size_t)h->perm[n]];
    tmp[2 * n + 1] = xy[2 * (size_t)h->perm[n] + 1];
  }
  if (cudaMemcpyAsync(h->d_pos, tmp.data(), h->V * 16, cudaMemcpyHostToDevice, h->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return GVIZ_CUDA_ERR_CUDA;
  return GVIZ_CUDA_OK;
}

int gvizCudaGripGetPositions(gvizCudaGrip *h, double *xy) {
  if (!h || (h->V && !xy)) return GVIZ_CUDA_ERR_ARG;
  GripGuard guard(h->device);
  if (!h->V) return GVIZ_CUDA_OK;
  std::vector<double> tmp(2 * h->V);
  if (cudaMemcpyAsync(tmp.data(), h->d_pos, h->V * 16, cudaMemcpyDeviceToHost, h->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return GVIZ_CUDA_ERR_CUDA;
  for (size_t n = 0; n < h->V; n++) {
    xy[2 * (size_t)h->perm[n]] = tmp[2 * n];
    xy[2 * (size_t)h->perm[n] + 1] = tmp[2 * n + 1];
  }
  return GVIZ_CUDA_OK;
}

int gvizCudaGripSetLayer(gvizCudaGrip *h, size_t layer, const uint32_t *active,
                         size_t activeCount, const uint64_t *knnOffsets,
                         const uint32_t *knnVertices, const uint32_t *knnDistances) {
  if (!h || activeCount > h->V || (activeCount && (!active || !knnOffsets)))
    return GVIZ_CUDA_ERR_ARG;
  const size_t K = activeCount ? knnOffsets[activeCount] : 0;
  if (K && (!knnVertices || !knnDistances)) return GVIZ_CUDA_ERR_ARG;
  for (size_t i = 0; i < activeCount; i++) {
    if (active[i] >= h->V || knnOffsets[i] > knnOffsets[i + 1]) return GVIZ_CUDA_ERR_ARG;
  }
  if (knnOffsets && activeCount && knnOffsets[0] != 0) return GVIZ_CUDA_ERR_ARG;
  for (size_t e = 0; e < K; e++)
    if (knnVertices[e] >= h->V) return GVIZ_CUDA_ERR_ARG;
  // the layer in labels (filtration order kept for the sums and the move);
  // the force kernel takes it in label order, its lists warp-interleaved:
  // entry e of list t = 32w + l at base[w] + 32e + l
  std::vector<uint32_t> act2(activeCount), order(activeCount), work(activeCount);
  for (size_t i = 0; i < activeCount; i++) {
    act2[i] = h->inv[active[i]];
    order[i] = (uint32_t)i;
  }
  std::sort(order.begin(), order.end(),
            [&](uint32_t x, uint32_t y) { return act2[x] < act2[y]; });
  std::vector<uint64_t> woff(activeCount + 1, 0);
  for (size_t t = 0; t < activeCount; t++) {
    work[t] = act2[order[t]];
    woff[t + 1] = woff[t] + (knnOffsets[order[t] + 1] - knnOffsets[order[t]]);
  }
  const size_t warps = (activeCount + 31) / 32;
  std::vector<uint64_t> base(warps + 1, 0);
  for (size_t w = 0; w < warps; w++) {
    uint64_t mx = 0;
    for (size_t t = 32 * w; t < activeCount && t < 32 * w + 32; t++)
      mx = std::max<uint64_t>(mx, woff[t + 1] - woff[t]);
    base[w + 1] = base[w] + 32 * mx;
  }
  const size_t T = base[warps];
  std::vector<uint32_t> iv(T, 0), id(T, 0);
  for (size_t t = 0; t < activeCount; t++) {
    const uint64_t b = base[t / 32] + (t % 32), src = knnOffsets[order[t]];
    for (uint64_t e = 0; e < woff[t + 1] - woff[t]; e++) {
      iv[b + 32 * e] = h->inv[knnVertices[src + e]];
      id[b + 32 * e] = knnDistances[src + e];
    }
  }
  GripGuard guard(h->device);
  if (T > h->knnCap) {
    cudaStreamSynchronize(h->stream);
    cudaFree(h->d_knnV);
    cudaFree(h->d_knnD);
    h->d_knnV = h->d_knnD = nullptr;
    h->knnCap = 0;
    if (galloc(&h->d_knnV, T) || galloc(&h->d_knnD, T)) return GVIZ_CUDA_ERR_ALLOC;
    h->knnCap = T;
  }
  h->n = activeCount;
  h->layer = layer;
  h->hasLayer = true;
  if (activeCount) {
    cudaMemcpyAsync(h->d_active, act2.data(), activeCount * 4, cudaMemcpyHostToDevice,
                    h->stream);
    cudaMemcpyAsync(h->d_work, work.data(), activeCount * 4, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->d_knnOff, woff.data(), (activeCount + 1) * 8, cudaMemcpyHostToDevice,
                    h->stream);
    cudaMemcpyAsync(h->d_warpBase, base.data(), (warps + 1) * 8, cudaMemcpyHostToDevice,
                    h->stream);
    if (T) {
      cudaMemcpyAsync(h->d_knnV, iv.data(), T * 4, cudaMemcpyHostToDevice, h->stream);
      cudaMemcpyAsync(h->d_knnD, id.data(), T * 4, cudaMemcpyHostToDevice, h->stream);
    }
  }
  if (h->V) cudaMemsetAsync(h->d_calc, 0, h->V, h->stream);
  if (activeCount) k_grip_clear<<<grid_for(activeCount), kThreads, 0, h->stream>>>(grip_args(h));
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return GVIZ_CUDA_ERR_CUDA;
  return GVIZ_CUDA_OK;
}

// everything of a round after the force kernel
void grip_after_forces(gvizCudaGrip *h, const GripArgs &a) {
  const uint32_t th = h->strict ? 1u : (uint32_t)kPartThreads;
  k_grip_part1<<<a.parts, th, 0, h->stream>>>(a);
  k_grip_final1<<<1, kPartThreads, 0, h->stream>>>(a);
  k_grip_part2<<<a.parts, th, 0, h->stream>>>(a);
  k_grip_final2<<<1, kPartThreads, 0, h->stream>>>(a);
  k_grip_apply<<<grid_for(h->n), kThreads, 0, h->stream>>>(a);
  k_grip_part3<<<a.parts, th, 0, h->stream>>>(a);
  k_grip_final3<<<1, kPartThreads, 0, h->stream>>>(a);
}

int gvizCudaGripRefineRound(gvizCudaGrip *h, gvizCudaGripRoundStats *stats) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  if (!h->hasLayer) return GVIZ_CUDA_ERR_NOT_BEGUN;
  GripGuard guard(h->device);
  double red[16] = {0};
  if (h->n) {
    const GripArgs a = grip_args(h);
    k_grip_pass1<<<grid_for(h->n), kThreads, 0, h->stream>>>(a);
    grip_after_forces(h, a);
    if (cudaGetLastError() != cudaSuccess) return GVIZ_CUDA_ERR_CUDA;
    if (cudaMemcpyAsync(red, h->d_red, sizeof red, cudaMemcpyDeviceToHost, h->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
      return GVIZ_CUDA_ERR_CUDA;
  }
  if (stats) {
    stats->maxDisplacement = red[6];
    stats->meanDisplacement = red[7];
    stats->meanHeat = red[8];
    stats->meanForce = red[9];
  }
  return GVIZ_CUDA_OK;
}

int gvizCudaGripTimeRounds(gvizCudaGrip *h, uint32_t rounds, float *totalMs, float *forcesMs) {
  if (!h || !totalMs) return GVIZ_CUDA_ERR_ARG;
  if (!h->hasLayer) return GVIZ_CUDA_ERR_NOT_BEGUN;
  GripGuard guard(h->device);
  *totalMs = 0.f;
  if (forcesMs) *forcesMs = 0.f;
  if (!h->n || !rounds) return GVIZ_CUDA_OK;
  std::vector<cudaEvent_t> ev(2 * (size_t)rounds + 2, nullptr);
  int rc = GVIZ_CUDA_OK;
  for (auto &e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) rc = GVIZ_CUDA_ERR_CUDA;
  if (!rc) {
    const GripArgs a = grip_args(h);
    cudaEventRecord(ev[0], h->stream);
    for (uint32_t r = 0; r < rounds; r++) {
      cudaEventRecord(ev[2 + 2 * r], h->stream);
      k_grip_pass1<<<grid_for(h->n), kThreads, 0, h->stream>>>(a);
      cudaEventRecord(ev[3 + 2 * r], h->stream);
      grip_after_forces(h, a);
    }
    cudaEventRecord(ev[1], h->stream);
    if (cudaEventSynchronize(ev[1]) != cudaSuccess ||
        cudaEventElapsedTime(totalMs, ev[0], ev[1]) != cudaSuccess)
      rc = GVIZ_CUDA_ERR_CUDA;
    float forces = 0.f;
    for (uint32_t r = 0; r < rounds && !rc; r++) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, ev[2 + 2 * r], ev[3 + 2 * r]) != cudaSuccess)
        rc = GVIZ_CUDA_ERR_CUDA;
      forces += t;
    }
    if (forcesMs) *forcesMs = forces;
  }
  for (auto &e : ev)
    if (e) cudaEventDestroy(e);
  return rc;
}

int gvizCudaGripGetDecorators(gvizCudaGrip *h, double *heat, double *disp, double *oldCos) {
  if (!h || (h->V && (!heat || !disp || !oldCos))) return GVIZ_CUDA_ERR_ARG;
  GripGuard guard(h->device);
  if (!h->V) return GVIZ_CUDA_OK;
  std::vector<double> th(h->V), td(2 * h->V), tc(h->V);
  cudaMemcpyAsync(th.data(), h->d_heat, h->V * 8, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(td.data(), h->d_disp, h->V * 16, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(tc.data(), h->d_oldCos, h->V * 8, cudaMemcpyDeviceToHost, h->stream);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return GVIZ_CUDA_ERR_CUDA;
  for (size_t n = 0; n < h->V; n++) {
    const size_t o = h->perm[n];
    heat[o] = th[n];
    disp[2 * o] = td[2 * n];
    disp[2 * o + 1] = td[2 * n + 1];
    oldCos[o] = tc[n];
  }
  return GVIZ_CUDA_OK;
}

}  // extern "C"
