// sort.cu -- hand-written device primitives: exclusive scan and a stable
// LSD radix sort of (uint64 key, uint32 value) pairs.
//
// The quadtree build sorts vertices by their quadrant path; stability keeps
// equal paths in vertex-index order, which is the arrival order of points in
// a reference leaf (src/ds/gvizQuadtree.c:129-131).
#include "internal.cuh"

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 2048
constexpr int kTopThreads = 1024;
constexpr int kTopItems = 8;  // top level handles 8192 tiles -> 16.7M entries

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;  // 4096 keys

// Block-wide exclusive scan of one value per thread; returns the block total.
template <int THREADS>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v,
                                                         uint32_t &excl) {
  __shared__ uint32_t warpTot[THREADS / 32];
  const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  uint32_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= (unsigned)o) inc += t;
  }
  if (lane == 31) warpTot[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint32_t t = lane < THREADS / 32 ? warpTot[lane] : 0;
    uint32_t ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t u = __shfl_up_sync(0xffffffffu, ti, o);
      if (lane >= (unsigned)o) ti += u;
    }
    if (lane < THREADS / 32) warpTot[lane] = ti - t;  // exclusive warp offsets
  }
  __syncthreads();
  excl = warpTot[w] + inc - v;
  __shared__ uint32_t blockTot;
  if (threadIdx.x == THREADS - 1) blockTot = excl + v;
  __syncthreads();
  uint32_t bt = blockTot;
  __syncthreads();
  return bt;
}

__global__ __launch_bounds__(kScanThreads) void k_scan_tiles(
    const uint32_t *__restrict__ in, uint32_t *out, uint32_t n,
    uint32_t *tileSums) {
  uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    uint32_t i = base + j;
    v[j] = i < n ? in[i] : 0u;
    s += v[j];
  }
  uint32_t excl;
  uint32_t tot = block_exclusive_scan<kScanThreads>(s, excl);
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    uint32_t i = base + j;
    if (i < n) out[i] = excl;
    excl += v[j];
  }
  if (threadIdx.x == 0) tileSums[blockIdx.x] = tot;
}

__global__ __launch_bounds__(kTopThreads) void k_scan_top(uint32_t *tileSums,
                                                          uint32_t nTiles,
                                                          uint32_t *total) {
  uint32_t per = (nTiles + kTopThreads - 1) / kTopThreads;
  uint32_t b = threadIdx.x * per;
  uint32_t s = 0;
  for (uint32_t j = 0; j < per; j++) {
    uint32_t i = b + j;
    if (i < nTiles) s += tileSums[i];
  }
  uint32_t excl;
  uint32_t tot = block_exclusive_scan<kTopThreads>(s, excl);
  for (uint32_t j = 0; j < per; j++) {
    uint32_t i = b + j;
    if (i < nTiles) {
      uint32_t t = tileSums[i];
      tileSums[i] = excl;
      excl += t;
    }
  }
  if (threadIdx.x == 0 && total) *total = tot;
}

// Whole scan in one block: each thread owns a contiguous run of ceil(n/1024)
// entries (n <= kSingleMax), one launch instead of three.
constexpr uint32_t kSingleMax = 1u << 13;  // one SM: only for small arrays

__global__ __launch_bounds__(kTopThreads) void k_scan_single(
    const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *total) {
  const uint32_t per = (n + kTopThreads - 1) / kTopThreads;
  const uint32_t b = threadIdx.x * per;
  uint32_t s = 0;
  for (uint32_t j = 0; j < per; j++) {
    const uint32_t i = b + j;
    if (i < n) s += in[i];
  }
  uint32_t excl;
  const uint32_t tot = block_exclusive_scan<kTopThreads>(s, excl);
  for (uint32_t j = 0; j < per; j++) {
    const uint32_t i = b + j;
    if (i < n) {
      const uint32_t t = in[i];
      out[i] = excl;
      excl += t;
    }
  }
  if (threadIdx.x == 0 && total) *total = tot;
}

__global__ void k_scan_add(uint32_t *out, uint32_t n,
                           const uint32_t *__restrict__ tileSums) {
  uint32_t add = tileSums[blockIdx.x];
  uint32_t base = blockIdx.x * kScanTile;
  for (uint32_t j = threadIdx.x; j < (uint32_t)kScanTile; j += blockDim.x) {
    uint32_t i = base + j;
    if (i < n) out[i] += add;
  }
}

__global__ __launch_bounds__(kSortThreads) void k_radix_hist(
    const uint64_t *__restrict__ keys, uint32_t n, int shift, uint32_t *hist,
    uint32_t numTiles) {
  __shared__ uint32_t sh[256];
  sh[threadIdx.x] = 0;
  __syncthreads();
  uint32_t base = blockIdx.x * kSortTile;
#pragma unroll 4
  for (int r = 0; r < kSortRounds; r++) {
    uint32_t i = base + r * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&sh[(uint32_t)(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * numTiles + blockIdx.x] = sh[threadIdx.x];
}

// Stable scatter: warp w of a tile owns 512 consecutive keys, taken in
// rounds of 32; __match_any_sync ranks equal digits inside a round.
// Shared memory of the scatter beyond its static arrays: the tile's keys
// and values reordered by digit.
constexpr size_t kScatterDyn = (size_t)kSortTile * (sizeof(uint64_t) + sizeof(uint32_t));

__global__ __launch_bounds__(kSortThreads) void k_radix_scatter(
    const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin,
    uint64_t *__restrict__ kout, uint32_t *__restrict__ vout, uint32_t n,
    int shift, const uint32_t *__restrict__ offs, uint32_t numTiles) {
  extern __shared__ __align__(16) unsigned char dyn[];
  uint64_t *sk = reinterpret_cast<uint64_t *>(dyn);
  uint32_t *sv = reinterpret_cast<uint32_t *>(sk + kSortTile);
  __shared__ uint32_t wcnt[kSortWarps][256];
  __shared__ uint32_t base[256];
  __shared__ uint32_t start[256];  // first in-tile position of each digit
  __shared__ uint32_t wsum[kSortWarps];
  const unsigned tid = threadIdx.x, w = tid >> 5, lane = tid & 31u;
  for (unsigned d = tid; d < kSortWarps * 256; d += kSortThreads)
    (&wcnt[0][0])[d] = 0;
  base[tid] = offs[tid * numTiles + blockIdx.x];
  __syncthreads();
  const uint32_t tileBase = blockIdx.x * kSortTile + w * (kSortRounds * 32);
  uint64_t k[kSortRounds];
  uint32_t v[kSortRounds];
  uint32_t rank[kSortRounds];
#pragma unroll
  for (int r = 0; r < kSortRounds; r++) {
    uint32_t i = tileBase + r * 32 + lane;
    bool valid = i < n;
    k[r] = valid ? kin[i] : 0ull;
    v[r] = valid ? vin[i] : 0u;
    uint32_t d = valid ? ((uint32_t)(k[r] >> shift) & 255u) : 256u;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t lt = peers & ((1u << lane) - 1u);
    uint32_t before = valid ? wcnt[w][d] : 0u;
    rank[r] = before + __popc(lt);
    __syncwarp();
    if (valid && lt == 0) wcnt[w][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // per digit (thread tid = digit): warps' offsets, then the tile's digit
  // starts by a block-wide exclusive scan of the digit totals
  uint32_t run = 0;
#pragma unroll
  for (int ww = 0; ww < kSortWarps; ww++) {
    uint32_t t = wcnt[ww][tid];
    wcnt[ww][tid] = run;
    run += t;
  }
  uint32_t incl = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (unsigned)o) incl += y;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  uint32_t before = 0;
  for (unsigned ww = 0; ww < w; ww++) before += wsum[ww];
  start[tid] = before + incl - run;
  __syncthreads();
  // the tile reordered by digit in shared memory (stable: warp, round, lane
  // is input order) ...
#pragma unroll
  for (int r = 0; r < kSortRounds; r++) {
    uint32_t i = tileBase + r * 32 + lane;
    if (i >= n) continue;
    uint32_t d = (uint32_t)(k[r] >> shift) & 255u;
    const uint32_t pos = start[d] + wcnt[w][d] + rank[r];
    sk[pos] = k[r];
    sv[pos] = v[r];
  }
  __syncthreads();
  // ... then written out in order: each digit's run lands contiguously
  const uint32_t t0 = blockIdx.x * kSortTile;
  const uint32_t cnt = n - t0 < (uint32_t)kSortTile ? n - t0 : (uint32_t)kSortTile;
  for (uint32_t j = tid; j < cnt; j += kSortThreads) {
    const uint64_t kk = sk[j];
    const uint32_t d = (uint32_t)(kk >> shift) & 255u;
    const uint32_t dst = base[d] + (j - start[d]);
    kout[dst] = kk;
    vout[dst] = sv[j];
  }
}

}  // namespace

size_t scan_scratch_entries(size_t n) {
  return (n + kScanTile - 1) / kScanTile + 1;
}

size_t radix_hist_entries(size_t n) {
  size_t tiles = (n + kSortTile - 1) / kSortTile;
  return 256 * (tiles ? tiles : 1);
}

// Exclusive scan of n uint32 (n <= 16.7M); in == out allowed. total may be
// nullptr or a device pointer receiving the sum.
void scan_exclusive(gvizCudaForce *h, const uint32_t *in, uint32_t *out,
                    size_t n, uint32_t *total) {
  if (n == 0) {
    if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), h->stream);
    return;
  }
  if (n <= kSingleMax) {
    k_scan_single<<<1, kTopThreads, 0, h->stream>>>(in, out, (uint32_t)n, total);
    return;
  }
  uint32_t tiles = (uint32_t)((n + kScanTile - 1) / kScanTile);
  k_scan_tiles<<<tiles, kScanThreads, 0, h->stream>>>(in, out, (uint32_t)n,
                                                      h->d_scanTile);
  k_scan_top<<<1, kTopThreads, 0, h->stream>>>(h->d_scanTile, tiles, total);
  if (tiles > 1)
    k_scan_add<<<tiles, 256, 0, h->stream>>>(out, (uint32_t)n, h->d_scanTile);
}

// Stable sort by the key bits above GVIZ_SORT_SKIP_BITS (an even number of
// 8-bit passes, so the result ends in (keys, vals)); keys equal in those bits
// keep their input order.
// The scatter's shared memory exceeds the default per-block budget: opted
// into once per device, at handle creation (outside any stream capture).
void sort_set_smem_limits() {
  cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kScatterDyn);
}

void radix_sort_pairs(gvizCudaForce *h, uint64_t *keys, uint32_t *vals,
                      uint64_t *keysAlt, uint32_t *valsAlt, size_t n) {
  if (n <= 1) return;
  uint32_t tiles = (uint32_t)((n + kSortTile - 1) / kSortTile);
  uint64_t *ka = keys, *kb = keysAlt;
  uint32_t *va = vals, *vb = valsAlt;
  for (int shift = GVIZ_SORT_SKIP_BITS; shift < 64; shift += 8) {
    k_radix_hist<<<tiles, kSortThreads, 0, h->stream>>>(ka, (uint32_t)n, shift,
                                                        h->d_radixHist, tiles);
    scan_exclusive(h, h->d_radixHist, h->d_radixHist, (size_t)256 * tiles,
                   nullptr);
    k_radix_scatter<<<tiles, kSortThreads, kScatterDyn, h->stream>>>(
        ka, va, kb, vb, (uint32_t)n, shift, h->d_radixHist, tiles);
    uint64_t *tk = ka;
    ka = kb;
    kb = tk;
    uint32_t *tv = va;
    va = vb;
    vb = tv;
  }
  prof_mark(h, "radix_sort");
}
