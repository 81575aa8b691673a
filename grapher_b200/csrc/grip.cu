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
constexpr int kSumThreads = 1024;

struct GripArgs {
  const uint64_t *row;
  const uint32_t *col;
  const uint32_t *active;
  const uint64_t *knnOff;
  const uint32_t *knnV, *knnD;
  double2 *pos, *disp, *oldDisp;
  double *heat, *oldCos, *lastF, *nrm;
  uint8_t *calc;
  double *red;  // [0,1] mean disp, [2,3] centroid, [4] omega, [5] rotate, [6..9] stats
  uint32_t n, layer;
};

// Spring forces (calculateSpringForces :892-934; the ops of
// include/core/gvizVec.h:138-316 via src/embedders/gvizForceDirected.c:6-20),
// then the heat update (:1071-1103 with updateLocalTemp :870-889) and the
// heat-scaled step.
__global__ __launch_bounds__(kThreads) void k_grip_pass1(GripArgs a) {
  const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= a.n) return;
  const uint32_t v = a.active[i];
  const double2 prev = a.disp[v];
  a.oldDisp[v] = prev;
  const double2 p = a.pos[v];
  double fx = 0.0, fy = 0.0;
  const uint64_t k0 = a.knnOff[i], k1 = a.knnOff[i + 1];
  if (a.layer > 0) {
    for (uint64_t e = k0; e < k1; e++) {  // KK springs at graph distance
      const double L = (double)a.knnD[e] * kEdge;
      if (L < 1e-9) continue;
      const double2 q = a.pos[a.knnV[e]];
      const double dx = q.x - p.x, dy = q.y - p.y;
      const double s = sqrt(dx * dx + dy * dy) / L - 1.0;
      fx += s * dx;
      fy += s * dy;
    }
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
    for (uint64_t e = k0; e < k1; e++) {  // from the k nearest
      const double2 q = a.pos[a.knnV[e]];
      const double dx = p.x - q.x, dy = p.y - q.y;
      const double d2 = dx * dx + dy * dy;
      if (d2 < 1e-18) continue;
      const double s = kFrScale * lenSq / d2;
      fx += s * dx;
      fy += s * dy;
    }
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

// Chunked ordered sums in one block (strict: one thread): thread t sums
// items [t*c, (t+1)*c) in order, thread 0 adds the chunk sums in order.
template <int K>
__device__ __forceinline__ void block_ordered_sum(double (&acc)[K], double (*part)[K]) {
  for (int k = 0; k < K; k++) part[threadIdx.x][k] = acc[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < K; k++) acc[k] = part[0][k];
    for (unsigned t = 1; t < blockDim.x; t++)
      for (int k = 0; k < K; k++) acc[k] += part[t][k];
  }
}

// mean displacement (removeNetTranslation :1106-1121) and centroid of the
// positions (removeNetRotation :1192-1203)
__global__ __launch_bounds__(kSumThreads) void k_grip_sums1(GripArgs a) {
  __shared__ double part[kSumThreads][4];
  const uint32_t c = (a.n + blockDim.x - 1) / blockDim.x;
  const uint32_t b = threadIdx.x * c, e = min(b + c, a.n);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t i = b; i < e; i++) {
    const uint32_t v = a.active[i];
    const double2 d = a.disp[v], p = a.pos[v];
    acc[0] += 1.0 * d.x;
    acc[1] += 1.0 * d.y;
    acc[2] += p.x;
    acc[3] += p.y;
  }
  block_ordered_sum<4>(acc, part);
  if (threadIdx.x == 0) {
    const double inv = 1.0 / (double)a.n;
    a.red[0] = acc[0] * inv;
    a.red[1] = acc[1] * inv;
    a.red[2] = acc[2] / (double)a.n;
    a.red[3] = acc[3] / (double)a.n;
  }
}

// angular momentum of the translated displacements and the polar moment of
// inertia about the centroid; omega = L / I (:1204-1252, dim 2)
__global__ __launch_bounds__(kSumThreads) void k_grip_sums2(GripArgs a) {
  __shared__ double part[kSumThreads][2];
  const uint32_t c = (a.n + blockDim.x - 1) / blockDim.x;
  const uint32_t b = threadIdx.x * c, e = min(b + c, a.n);
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
  block_ordered_sum<2>(acc, part);
  if (threadIdx.x == 0) {
    const bool rotate = a.n >= 3 && !(fabs(acc[1]) < kEps);
    a.red[4] = rotate ? acc[0] / acc[1] : 0.0;
    a.red[5] = rotate ? 1.0 : 0.0;
  }
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
__global__ __launch_bounds__(kSumThreads) void k_grip_stats(GripArgs a) {
  __shared__ double part[kSumThreads][4];
  const uint32_t c = (a.n + blockDim.x - 1) / blockDim.x;
  const uint32_t b = threadIdx.x * c, e = min(b + c, a.n);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};  // max, sum disp, sum heat, sum force
  for (uint32_t i = b; i < e; i++) {
    const uint32_t v = a.active[i];
    const double nrm = a.nrm[i];
    if (nrm > acc[0]) acc[0] = nrm;
    acc[1] += nrm;
    acc[2] += a.heat[v];
    acc[3] += a.lastF[v];
  }
  part[threadIdx.x][0] = acc[0];
  __syncthreads();
  double mx = acc[0];
  if (threadIdx.x == 0)
    for (unsigned t = 1; t < blockDim.x; t++) mx = fmax(mx, part[t][0]);
  __syncthreads();
  block_ordered_sum<4>(acc, part);
  if (threadIdx.x == 0) {
    a.red[6] = mx;
    a.red[7] = a.n ? acc[1] / a.n : 0.0;
    a.red[8] = a.n ? acc[2] / a.n : 0.0;
    a.red[9] = a.n ? acc[3] / a.n : 0.0;
  }
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
  uint64_t *d_knnOff = nullptr;
  size_t n = 0, knnCap = 0, layer = 0;
  bool hasLayer = false;
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
  a.knnOff = h->d_knnOff;
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
  if (rc) {
    grip_free(h);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return rc;
  }
  if (V) {
    cudaMemcpyAsync(h->d_row, rowOffsets, (V + 1) * 8, cudaMemcpyHostToDevice, h->stream);
    if (E2) cudaMemcpyAsync(h->d_col, neighbors, E2 * 4, cudaMemcpyHostToDevice, h->stream);
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
  if (cudaMemcpyAsync(h->d_pos, xy, h->V * 16, cudaMemcpyHostToDevice, h->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return GVIZ_CUDA_ERR_CUDA;
  return GVIZ_CUDA_OK;
}

int gvizCudaGripGetPositions(gvizCudaGrip *h, double *xy) {
  if (!h || (h->V && !xy)) return GVIZ_CUDA_ERR_ARG;
  GripGuard guard(h->device);
  if (!h->V) return GVIZ_CUDA_OK;
  if (cudaMemcpyAsync(xy, h->d_pos, h->V * 16, cudaMemcpyDeviceToHost, h->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return GVIZ_CUDA_ERR_CUDA;
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
  GripGuard guard(h->device);
  if (K > h->knnCap) {
    cudaStreamSynchronize(h->stream);
    cudaFree(h->d_knnV);
    cudaFree(h->d_knnD);
    h->d_knnV = h->d_knnD = nullptr;
    h->knnCap = 0;
    if (galloc(&h->d_knnV, K) || galloc(&h->d_knnD, K)) return GVIZ_CUDA_ERR_ALLOC;
    h->knnCap = K;
  }
  h->n = activeCount;
  h->layer = layer;
  h->hasLayer = true;
  if (activeCount) {
    cudaMemcpyAsync(h->d_active, active, activeCount * 4, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->d_knnOff, knnOffsets, (activeCount + 1) * 8, cudaMemcpyHostToDevice,
                    h->stream);
    if (K) {
      cudaMemcpyAsync(h->d_knnV, knnVertices, K * 4, cudaMemcpyHostToDevice, h->stream);
      cudaMemcpyAsync(h->d_knnD, knnDistances, K * 4, cudaMemcpyHostToDevice, h->stream);
    }
  }
  if (h->V) cudaMemsetAsync(h->d_calc, 0, h->V, h->stream);
  if (activeCount) k_grip_clear<<<grid_for(activeCount), kThreads, 0, h->stream>>>(grip_args(h));
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return GVIZ_CUDA_ERR_CUDA;
  return GVIZ_CUDA_OK;
}

int gvizCudaGripRefineRound(gvizCudaGrip *h, gvizCudaGripRoundStats *stats) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  if (!h->hasLayer) return GVIZ_CUDA_ERR_NOT_BEGUN;
  GripGuard guard(h->device);
  double red[16] = {0};
  if (h->n) {
    const GripArgs a = grip_args(h);
    const uint32_t sumThreads = h->strict ? 1u : (uint32_t)kSumThreads;
    k_grip_pass1<<<grid_for(h->n), kThreads, 0, h->stream>>>(a);
    k_grip_sums1<<<1, sumThreads, 0, h->stream>>>(a);
    k_grip_sums2<<<1, sumThreads, 0, h->stream>>>(a);
    k_grip_apply<<<grid_for(h->n), kThreads, 0, h->stream>>>(a);
    k_grip_stats<<<1, sumThreads, 0, h->stream>>>(a);
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

int gvizCudaGripGetDecorators(gvizCudaGrip *h, double *heat, double *disp, double *oldCos) {
  if (!h || (h->V && (!heat || !disp || !oldCos))) return GVIZ_CUDA_ERR_ARG;
  GripGuard guard(h->device);
  if (!h->V) return GVIZ_CUDA_OK;
  cudaMemcpyAsync(heat, h->d_heat, h->V * 8, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(disp, h->d_disp, h->V * 16, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(oldCos, h->d_oldCos, h->V * 8, cudaMemcpyDeviceToHost, h->stream);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return GVIZ_CUDA_ERR_CUDA;
  return GVIZ_CUDA_OK;
}

}  // extern "C"
