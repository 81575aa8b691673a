// noalloc.cu -- an allocation-free variant of the ForceAtlas2 global speed
// update (the swing/traction reduction of precise.cu's k_fa2_chunks and the
// speed rule of k_fa2_speed), for callers that must not allocate device
// memory while they run.
//
// Who needs it: a render loop that calls the layout once per frame and is not
// allowed to touch the device allocator inside the frame (a cudaMalloc can
// synchronise the device and stall the frame), and host programs whose device
// memory is owned by another allocator (a framework's caching pool that has
// already reserved the GPU), where a library-side cudaMalloc may fail or
// fragment that pool. Such callers compute structForce with their own kernels
// and only want the reference's adaptive speed (updateGlobalSpeed,
// src/embedders/gvizForceEmbedder.c:140-185) applied to it.
//
// The per-chunk partial sums that the handle-based path keeps in a buffer
// allocated by gvizCudaForceCreate live here in one file-scope device array of
// GVIZ_NOALLOC_MAX_CHUNKS * 2 doubles (64 KiB), which every GPU that loads the
// library holds until the process exits.
//
// Compiled with --fmad=false like precise.cu, and the partial sums are added
// in the same order as the handle-based step's (per chunk a strided loop and
// a block reduction, then over the chunks a strided loop and a block
// reduction), so for one layout the results are bit-identical to the
// handle-based FP64 step for the same inputs.
#include <math.h>

#include <atomic>

#include "internal.cuh"

#define GVIZ_NOALLOC_MAX_CHUNKS 4096  // -> at most 4096 * 2048 vertices

namespace {

constexpr int kThreads = 256;

// Shared by every call on a device. Each call writes every slot it later
// reads (chunks [0, nChunks)), so nothing has to start at zero; two calls
// that overlap on the GPU (different streams, no ordering) race on it.
static __device__ __align__(256) double g_speedScratch[2 * GVIZ_NOALLOC_MAX_CHUNKS];

__device__ __forceinline__ double block_sum_na(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31u) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kThreads / 32; w++) r += sh[w];
  __syncthreads();
  return r;
}

// swing_i = m_i |f - f_old|, traction_i = m_i * 0.5 |f + f_old|
// (src/embedders/gvizForceEmbedder.c:128-138), per-chunk sums into scratch.
__global__ __launch_bounds__(kThreads) void k_na_swing(
    const double2 *__restrict__ sf, const double2 *__restrict__ sfOld,
    const double *__restrict__ mass, uint32_t n, double *swingOut,
    double *scratch) {
  __shared__ double sh[kThreads / 32];
  const uint32_t c = blockIdx.x;
  const uint32_t b = c * GVIZ_CHUNK;
  const uint32_t e = min(b + (uint32_t)GVIZ_CHUNK, n);
  double sw = 0.0, tr = 0.0;
  for (uint32_t v = b + threadIdx.x; v < e; v += kThreads) {
    const double2 f = sf[v], o = sfOld[v];
    const double m = mass[v];
    const double d0 = f.x - o.x, d1 = f.y - o.y;
    const double s0 = f.x + o.x, s1 = f.y + o.y;
    const double swing = m * sqrt(d0 * d0 + d1 * d1);
    const double trac = m * 0.5 * sqrt(s0 * s0 + s1 * s1);
    if (swingOut) swingOut[v] = swing;
    sw += swing;
    tr += trac;
  }
  sw = block_sum_na(sw, sh);
  tr = block_sum_na(tr, sh);
  if (threadIdx.x == 0) {
    scratch[2 * c] = sw;
    scratch[2 * c + 1] = tr;
  }
}

// updateGlobalSpeed on the chunk partials: one block, thread t adds chunks
// t, t + kThreads, ..., then the block reduction (the order of k_fa2_speed).
__global__ __launch_bounds__(kThreads) void k_na_speed(const double *scratch, uint32_t nChunks,
                                                        uint32_t n, double jitterTolerance,
                                                        double *state) {
  __shared__ double sh[kThreads / 32];
  double totalSwing = 0.0, totalTraction = 0.0;
  for (uint32_t c = threadIdx.x; c < nChunks; c += kThreads) {
    totalSwing += scratch[2 * c];
    totalTraction += scratch[2 * c + 1];
  }
  totalSwing = block_sum_na(totalSwing, sh);
  totalTraction = block_sum_na(totalTraction, sh);
  if (threadIdx.x != 0) return;
  if (totalTraction < 1e-7) return;
  double speed = state[0], eff = state[1];
  const double nn = (double)n;
  const double estimatedOptimalJT = 0.05 * sqrt(nn);
  const double minJT = sqrt(estimatedOptimalJT);
  const double maxJT = 10.0;
  double jt = jitterTolerance *
              fmax(minJT, fmin(maxJT, estimatedOptimalJT * totalTraction / (nn * nn)));
  if (totalSwing / totalTraction > 2.0) {
    if (eff > 0.05) eff *= 0.5;
    jt = fmax(jt, jitterTolerance);
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
  state[0] = speed;
  state[1] = eff;
}

// Device address of g_speedScratch per device ordinal, looked up once with
// that device current and kept for the life of the process (atomics: first
// calls from several host threads may race to store it; they store the same
// value). The name g_speedScratch in host code is only a host-side stand-in
// and must never be passed to a kernel.
std::atomic<double *> g_scratchAddr[64];

}  // namespace

extern "C" int gvizCudaFa2SpeedUpdateNoAlloc(
    const double *d_structForce, const double *d_oldStructForce,
    const double *d_mass, size_t vertexCount, double jitterTolerance,
    double *d_swing, double *d_speedState, void *stream) {
  if (!d_speedState || (vertexCount && (!d_structForce || !d_oldStructForce || !d_mass)))
    return GVIZ_CUDA_ERR_ARG;
  const size_t nChunks = (vertexCount + GVIZ_CHUNK - 1) / GVIZ_CHUNK;
  if (nChunks > GVIZ_NOALLOC_MAX_CHUNKS) return GVIZ_CUDA_ERR_LIMIT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return GVIZ_CUDA_ERR_NO_DEVICE;
  double *scratch = g_scratchAddr[dev].load(std::memory_order_acquire);
  if (!scratch) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_speedScratch) != cudaSuccess || !p)
      return GVIZ_CUDA_ERR_CUDA;
    scratch = static_cast<double *>(p);
    g_scratchAddr[dev].store(scratch, std::memory_order_release);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (nChunks)
    k_na_swing<<<(unsigned)nChunks, kThreads, 0, st>>>(
        reinterpret_cast<const double2 *>(d_structForce),
        reinterpret_cast<const double2 *>(d_oldStructForce), d_mass,
        (uint32_t)vertexCount, d_swing, scratch);
  k_na_speed<<<1, kThreads, 0, st>>>(scratch, (uint32_t)nChunks, (uint32_t)vertexCount,
                                     jitterTolerance, d_speedState);
  return cudaGetLastError() == cudaSuccess ? GVIZ_CUDA_OK : GVIZ_CUDA_ERR_CUDA;
}
