// sort.cu -- hand-written device primitives: exclusive scan and a stable
// LSD radix sort of (uint64 key, uint32 value) pairs.
//
// The quadtree build sorts vertices by their quadrant path; stability keeps
// equal paths in vertex-index order, which is the arrival order of points in
// a reference leaf (src/ds/gvizQuadtree.c:129-131).
//
// Both are single-pass over their input per digit (per scan): a tile takes
// its index from a ticket counter, so every lower tile has started before
// it; it publishes its count (flag AGGREGATE), then adds the counts of the
// tiles before it, walking back until one has published its inclusive
// prefix (flag PREFIX), and publishes its own prefix (decoupled look-back).
// The first pass's digit counts come from one read of the keys; each pass
// counts the next pass's digits of the keys it holds.
// Status words are 64 bits (flag in the high half, count in the low half),
// written and read with single relaxed accesses; a wait that outlasts its
// iteration limit sets GVIZ_ST_TREE and ends.
#include <algorithm>

#include "internal.cuh"

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 2048
constexpr int kTopThreads = 1024;

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;  // 4096 keys
constexpr int kSortPasses = (64 - GVIZ_SORT_SKIP_BITS) / 8;
static_assert(kSortPasses % 2 == 0, "the sorted pairs must end in the input buffers");

constexpr uint64_t kFlagAggregate = 1ull << 32;
constexpr uint64_t kFlagPrefix = 2ull << 32;
constexpr uint32_t kLookbackSpin = 1u << 22;  // reads of a status word before giving up

__device__ __forceinline__ uint64_t ld_status(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_status(uint64_t *p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// The sum of the counts of tiles [0, tile) in the status column `st` of
// stride `stride` (tile t's word is st[t * stride]), read kLookbackWidth
// tiles at a time (independent loads). Tile 0 publishes its prefix without
// waiting, so the walk always ends.
constexpr int kLookbackWidth = 8;

__device__ __forceinline__ uint32_t lookback(const uint64_t *st, size_t stride, uint32_t tile,
                                             uint32_t *status) {
  uint32_t excl = 0;
  uint32_t spins = 0;
  for (int64_t p = (int64_t)tile - 1; p >= 0; p -= kLookbackWidth) {
    uint64_t w[kLookbackWidth];
#pragma unroll
    for (int i = 0; i < kLookbackWidth; i++)
      w[i] = p - i >= 0 ? ld_status(st + (size_t)(p - i) * stride) : kFlagPrefix;
#pragma unroll
    for (int i = 0; i < kLookbackWidth; i++) {
      while ((w[i] >> 32) == 0) {  // not published yet
        if (++spins > kLookbackSpin) {
          atomicOr(status, GVIZ_ST_TREE);
          return excl;
        }
        w[i] = ld_status(st + (size_t)(p - i) * stride);
      }
      excl += (uint32_t)w[i];
      if ((w[i] & ~0xffffffffull) == kFlagPrefix) return excl;
    }
  }
  return excl;
}

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

// Single-pass exclusive scan: tile = ticket, 2048 entries per tile.
// state: [0] ticket, [1 + t] status of tile t.
__global__ __launch_bounds__(kScanThreads) void k_scan_onepass(
    const uint32_t *in, uint32_t *out, uint32_t n, uint64_t *state, uint32_t *total,
    uint32_t *status) {
  __shared__ uint32_t sTile, sExcl;
  if (threadIdx.x == 0) sTile = atomicAdd(reinterpret_cast<unsigned long long *>(state), 1ull);
  __syncthreads();
  const uint32_t tile = sTile;
  const uint32_t base = tile * kScanTile + threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const uint32_t i = base + j;
    v[j] = i < n ? in[i] : 0u;
    s += v[j];
  }
  uint32_t excl;
  const uint32_t tot = block_exclusive_scan<kScanThreads>(s, excl);
  uint64_t *st = state + 1;
  if (threadIdx.x == 0) {
    if (tile == 0) {
      st_status(st, kFlagPrefix | tot);
      sExcl = 0;
    } else {
      st_status(st + tile, kFlagAggregate | tot);
      const uint32_t before = lookback(st, 1, tile, status);
      st_status(st + tile, kFlagPrefix | (before + tot));
      sExcl = before;
    }
    const uint32_t nTiles = (n + kScanTile - 1) / kScanTile;
    if (total && tile == nTiles - 1) *total = sExcl + tot;
  }
  __syncthreads();
  excl += sExcl;
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const uint32_t i = base + j;
    if (i < n) out[i] = excl;
    excl += v[j];
  }
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

// Digit counts of the first sort pass (each later pass counts the digit of
// the pass after it while it scatters).
__global__ __launch_bounds__(kSortThreads) void k_radix_hist0(
    const uint64_t *__restrict__ keys, uint32_t n, uint32_t *ghist) {
  __shared__ uint32_t sh[256];
  sh[threadIdx.x] = 0u;
  __syncthreads();
  const uint32_t stride = gridDim.x * kSortThreads;
  for (uint32_t i = blockIdx.x * kSortThreads + threadIdx.x; i < n; i += stride)
    atomicAdd(&sh[(uint32_t)(keys[i] >> GVIZ_SORT_SKIP_BITS) & 255u], 1u);
  __syncthreads();
  const uint32_t c = sh[threadIdx.x];
  if (c) atomicAdd(ghist + threadIdx.x, c);
}

// Stable scatter: warp w of a tile owns 512 consecutive keys, taken in
// rounds of 32; __match_any_sync ranks equal digits inside a round.
// Shared memory of the scatter beyond its static arrays: the tile's keys
// and values reordered by digit.
constexpr size_t kScatterDyn = (size_t)kSortTile * (sizeof(uint64_t) + sizeof(uint32_t));

// One pass over digit `pass`: tile = ticket; each digit's start in the
// output is its global start (a scan of ghist) plus its count in the tiles
// before (look-back over the status words state[tile * 256 + digit]).
__global__ __launch_bounds__(kSortThreads) void k_radix_onesweep(
    const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin,
    uint64_t *__restrict__ kout, uint32_t *__restrict__ vout, uint32_t n,
    int pass, uint32_t *ghist, uint64_t *state, uint32_t *ticket,
    uint32_t *status) {
  extern __shared__ __align__(16) unsigned char dyn[];
  uint64_t *sk = reinterpret_cast<uint64_t *>(dyn);
  uint32_t *sv = reinterpret_cast<uint32_t *>(sk + kSortTile);
  __shared__ uint32_t wcnt[kSortWarps][256];
  __shared__ uint32_t base[256];
  __shared__ uint32_t start[256];  // first in-tile position of each digit
  __shared__ uint32_t wsum[kSortWarps];
  __shared__ uint32_t sTile;
  __shared__ uint32_t nextCnt[256];  // the next pass's digit counts of this tile
  const unsigned tid = threadIdx.x, w = tid >> 5, lane = tid & 31u;
  const int shift = GVIZ_SORT_SKIP_BITS + 8 * pass;
  const bool countNext = pass + 1 < kSortPasses;
  if (tid == 0) sTile = atomicAdd(ticket, 1u);
  for (unsigned d = tid; d < kSortWarps * 256; d += kSortThreads)
    (&wcnt[0][0])[d] = 0;
  nextCnt[tid] = 0u;
  // the digit's first output position: exclusive scan of the global counts
  uint32_t gstart;
  block_exclusive_scan<kSortThreads>(ghist[pass * 256 + tid], gstart);
  __syncthreads();
  const uint32_t tile = sTile;
  const uint32_t tileBase = tile * kSortTile + w * (kSortRounds * 32);
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
    if (countNext && valid) atomicAdd(&nextCnt[(uint32_t)(k[r] >> (shift + 8)) & 255u], 1u);
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
  // this tile's count of digit tid, then the counts of the tiles before
  {
    uint64_t *col = state + tid;
    if (tile == 0) {
      st_status(col, kFlagPrefix | run);
      base[tid] = gstart;
    } else {
      st_status(col + (size_t)tile * 256, kFlagAggregate | run);
      const uint32_t before = lookback(col, 256, tile, status);
      st_status(col + (size_t)tile * 256, kFlagPrefix | (before + run));
      base[tid] = gstart + before;
    }
  }
  if (countNext && nextCnt[tid]) atomicAdd(ghist + (pass + 1) * 256 + tid, nextCnt[tid]);
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
  const uint32_t t0 = tile * kSortTile;
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

size_t scan_state_entries(size_t n) {
  return (n + kScanTile - 1) / kScanTile + 1;
}

size_t sort_state_entries(size_t n) {
  const size_t tiles = (n + kSortTile - 1) / kSortTile;
  // per pass: tiles * 256 status words; then the global counts (uint32) and
  // the tickets, in 64-bit words
  return (size_t)kSortPasses * 256 * (tiles ? tiles : 1) + kSortPasses * 128 + kSortPasses;
}

// Exclusive scan of n uint32 (n <= 2^31); in == out allowed. total may be
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
  const uint32_t tiles = (uint32_t)((n + kScanTile - 1) / kScanTile);
  cudaMemsetAsync(h->d_scanState, 0, (tiles + 1) * sizeof(uint64_t), h->stream);
  k_scan_onepass<<<tiles, kScanThreads, 0, h->stream>>>(in, out, (uint32_t)n, h->d_scanState,
                                                        total, h->d_status);
}

// Stable sort by the key bits above GVIZ_SORT_SKIP_BITS (an even number of
// 8-bit passes, so the result ends in (keys, vals)); keys equal in those bits
// keep their input order.
// The scatter's shared memory exceeds the default per-block budget: opted
// into once per device, at handle creation (outside any stream capture).
void sort_set_smem_limits() {
  cudaFuncSetAttribute(k_radix_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kScatterDyn);
}

void radix_sort_pairs(gvizCudaForce *h, uint64_t *keys, uint32_t *vals,
                      uint64_t *keysAlt, uint32_t *valsAlt, size_t n) {
  if (n <= 1) return;
  const uint32_t tiles = (uint32_t)((n + kSortTile - 1) / kSortTile);
  uint64_t *state = h->d_sortState;
  const size_t statusWords = (size_t)kSortPasses * 256 * tiles;
  uint32_t *ghist = reinterpret_cast<uint32_t *>(state + statusWords);
  uint32_t *tickets = ghist + kSortPasses * 256;
  cudaMemsetAsync(state, 0, (statusWords + kSortPasses * 128 + kSortPasses) * sizeof(uint64_t),
                  h->stream);
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint32_t hb = std::min<uint32_t>(tiles * 4u, (uint32_t)(sms > 0 ? sms : 1) * 2u);
  k_radix_hist0<<<hb, kSortThreads, 0, h->stream>>>(keys, (uint32_t)n, ghist);
  uint64_t *ka = keys, *kb = keysAlt;
  uint32_t *va = vals, *vb = valsAlt;
  for (int pass = 0; pass < kSortPasses; pass++) {
    k_radix_onesweep<<<tiles, kSortThreads, kScatterDyn, h->stream>>>(
        ka, va, kb, vb, (uint32_t)n, pass, ghist, state + (size_t)pass * 256 * tiles,
        tickets + pass, h->d_status);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  prof_mark(h, "radix_sort");
}
