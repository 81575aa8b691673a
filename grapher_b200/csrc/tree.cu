// tree.cu -- device rebuild of gviz's quadtree (src/ds/gvizQuadtree.c) as a
// compressed, preorder-laid-out tree whose leaves hold exactly the point
// sets of the reference's leaves.
//
// Pipeline (one launch each, no host synchronisation):
//   bbox per chunk -> square root box per graph (gvizQuadtree.c:165-178)
//   per point: quadrant path by replaying the reference's FP64 descent
//     (QuadrantFor :65-73 against centres cx +/- halfSize/2, Subdivide :75-92)
//   stable radix sort of (graph, path) -> fix-up sort of equal-prefix runs
//   buckets = identical full paths -> Karras binary radix tree (2012)
//   binary nodes merged into quadtree nodes (two path bits per level)
//   bottom-up mass / centre-of-mass / subtree sizes (arrival counters):
//     inside blocks of 256 buckets through shared memory, then the few
//     nodes spanning blocks on a persistent grid
//   preorder index of the spanning nodes by walking up weighted parent
//   links, then every node record, its own walk up stopping at the first
//   spanning ancestor
//
// Why the compressed tree walks like the reference's: a chain of single-child
// nodes shares one point set, hence one mass and centre of mass; the
// reference accepts some chain node iff it accepts the deepest one (the
// ratio only shrinks going down), so one node per chain, tested with the
// deepest chain halfSize, gives the same pseudo-bodies. Leaves are never
// tested (gvizForceEmbedder.c:41-53); an overflow leaf below a chain is
// tested with its parent's halfSize. Empty children are skipped there too
// (mass == 0, :38-39).
#include <math.h>

#include <algorithm>

#include <cuda/atomic>

#include "internal.cuh"

namespace {

constexpr int kThreads = 256;


// ---------------------------------------------------------------------------
// bounding boxes and roots
// ---------------------------------------------------------------------------

__global__ __launch_bounds__(kThreads) void k_bbox_chunks(
    const double2 *__restrict__ pos, const uint32_t *__restrict__ cb,
    const uint32_t *__restrict__ ce, double4 *box, uint32_t *status) {
  const uint32_t b = cb[blockIdx.x], e = ce[blockIdx.x];
  double mnx = INFINITY, mxx = -INFINITY, mny = INFINITY, mxy = -INFINITY;
  int bad = 0;
  for (uint32_t i = b + threadIdx.x; i < e; i += kThreads) {
    double2 p = pos[i];
    if (!isfinite(p.x) || !isfinite(p.y)) bad = 1;
    mnx = fmin(mnx, p.x);
    mxx = fmax(mxx, p.x);
    mny = fmin(mny, p.y);
    mxy = fmax(mxy, p.y);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mnx = fmin(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
    mxx = fmax(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
    mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    mxy = fmax(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
  }
  __shared__ double4 wb[kThreads / 32];
  if (lane_id() == 0) wb[threadIdx.x >> 5] = make_double4(mnx, mxx, mny, mxy);
  if (bad) atomicOr(status, GVIZ_ST_NONFINITE);
  __syncthreads();
  if (threadIdx.x == 0) {
    double4 r = wb[0];
    for (int w = 1; w < kThreads / 32; w++) {
      r.x = fmin(r.x, wb[w].x);
      r.y = fmax(r.y, wb[w].y);
      r.z = fmin(r.z, wb[w].z);
      r.w = fmax(r.w, wb[w].w);
    }
    box[blockIdx.x] = r;
  }
}

// One block per graph: min/max over the graph's chunk boxes (order-free, so
// exact), then the root box of gvizQuadtreeBuild.
__global__ __launch_bounds__(kThreads) void k_graph_roots(
    const double4 *__restrict__ box, const uint32_t *__restrict__ gcb,
    const uint32_t *__restrict__ gce, GraphRoot *roots, uint32_t G,
    uint32_t *status) {
  const uint32_t g = blockIdx.x;
  double mnx = INFINITY, mxx = -INFINITY, mny = INFINITY, mxy = -INFINITY;
  for (uint32_t c = gcb[g] + threadIdx.x; c < gce[g]; c += kThreads) {
    double4 r = box[c];
    mnx = fmin(mnx, r.x);
    mxx = fmax(mxx, r.y);
    mny = fmin(mny, r.z);
    mxy = fmax(mxy, r.w);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mnx = fmin(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
    mxx = fmax(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
    mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    mxy = fmax(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
  }
  __shared__ double4 wb[kThreads / 32];
  if (lane_id() == 0) wb[threadIdx.x >> 5] = make_double4(mnx, mxx, mny, mxy);
  __syncthreads();
  if (threadIdx.x != 0) return;
  for (int w = 1; w < kThreads / 32; w++) {
    mnx = fmin(mnx, wb[w].x);
    mxx = fmax(mxx, wb[w].y);
    mny = fmin(mny, wb[w].z);
    mxy = fmax(mxy, wb[w].w);
  }
  mnx = fmin(mnx, wb[0].x);
  mxx = fmax(mxx, wb[0].y);
  mny = fmin(mny, wb[0].z);
  mxy = fmax(mxy, wb[0].w);
  GraphRoot R;
  if (!(mnx <= mxx)) {  // empty graph
    R.cx = 0.0;
    R.cy = 0.0;
    R.h0 = 1.0;
    R.D = 0;
    R.capped = 0;
    roots[g] = R;
    return;
  }
  double sx = mxx - mnx, sy = mxy - mny;
  double span = sx > sy ? sx : sy;
  R.h0 = span > 0.0 ? span / 2.0 : 1.0;
  R.cx = (mnx + mxx) / 2.0;
  R.cy = (mny + mxy) / 2.0;
  double h = R.h0;
  int d = 0;
  while (h > 1e-9 && d < 64) {
    h = h / 2.0;
    d++;
  }
  R.D = d;
  R.capped = h > 1e-9 ? 1 : 0;
  if (R.capped) atomicOr(status, GVIZ_ST_DEPTH_CAP);
  roots[g] = R;
}

// Quadrant path of every point: digit = (north ? 0 : 2) + (east ? 1 : 0),
// i.e. NW=0 NE=1 SW=2 SE=3 (include/ds/gvizQuadtree.h:11-17), so sorted
// paths are the reference's depth-first NW,NE,SW,SE order.
__global__ __launch_bounds__(kThreads) void k_keys(
    const double2 *__restrict__ pos, const uint32_t *__restrict__ gid,
    const GraphRoot *__restrict__ roots, uint64_t *keyHi, uint64_t *keyLo,
    uint64_t *ck, uint32_t *idx, uint32_t V, int gbits) {
  uint32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= V) return;
  const uint32_t g = gid ? gid[i] : 0u;
  const GraphRoot R = roots[g];
  const double2 p = pos[i];
  double cx = R.cx, cy = R.cy, h = R.h0;
  uint64_t hi = 0, lo = 0;
  for (int d = 1; d <= R.D; d++) {
    const bool east = p.x >= cx;
    const bool north = p.y >= cy;
    const uint64_t q = (north ? 0ull : 2ull) | (east ? 1ull : 0ull);
    const double quarter = h / 2.0;
    cx = east ? cx + quarter : cx + (-quarter);
    cy = north ? cy + quarter : cy + (-quarter);
    h = quarter;
    if (d <= 32)
      hi |= q << (64 - 2 * d);
    else
      lo |= q << (128 - 2 * d);
  }
  keyHi[i] = hi;
  keyLo[i] = lo;
  ck[i] = gbits ? (((uint64_t)g << (64 - gbits)) | (hi >> gbits)) : hi;
  idx[i] = i;
}

// The sorted points' full paths, and the starts of runs of equal composite
// keys (the sorted bits of the composite key).
__global__ __launch_bounds__(kThreads) void k_gather_keys(
    const uint32_t *__restrict__ idx, const uint64_t *__restrict__ keyHi,
    const uint64_t *__restrict__ keyLo, const uint64_t *__restrict__ ck, uint64_t *sHi,
    uint64_t *sLo, uint32_t *flag, uint32_t V) {
  uint32_t s = blockIdx.x * kThreads + threadIdx.x;
  if (s >= V) return;
  uint32_t i = idx[s];
  sHi[s] = keyHi[i];
  sLo[s] = keyLo[i];
  flag[s] = (s == 0 || (ck[s] >> GVIZ_SORT_SKIP_BITS) !=
                           (ck[s - 1] >> GVIZ_SORT_SKIP_BITS)) ? 1u : 0u;
}

// ---------------------------------------------------------------------------
// runs of equal composite keys
// ---------------------------------------------------------------------------

// Runs of equal composite keys (equal sorted prefixes). The thread at a
// run's start finds its end, the first later key whose sorted prefix
// differs, by a galloping search over the sorted keys (most runs are one
// key long, found by the first probe). Runs longer than the leaf capacity k
// need their deeper digits sorted; runs of 2..k points lie in one leaf, so
// their keys are cut to the common prefix (the leaf keeps them in vertex
// order, as the reference does).
__global__ __launch_bounds__(kThreads) void k_runs(
    const uint64_t *__restrict__ ck, const uint32_t *__restrict__ flag, uint32_t *counts,
    uint32_t *deep, uint64_t *sHi, uint64_t *sLo, uint32_t V, uint32_t k, int gbits) {
  const uint32_t start = blockIdx.x * kThreads + threadIdx.x;
  if (start >= V || !flag[start]) return;
  const uint64_t key = ck[start] >> GVIZ_SORT_SKIP_BITS;
  uint32_t end = start + 1u;
  if (end < V && (ck[end] >> GVIZ_SORT_SKIP_BITS) == key) {
    uint32_t lo = end, hi = V;  // ck[lo] is in the run, the end is in (lo, hi]
    for (uint32_t step = 1u;; step <<= 1) {
      const uint32_t probe = lo + step;
      if (probe >= V || probe < lo) break;
      if ((ck[probe] >> GVIZ_SORT_SKIP_BITS) != key) {
        hi = probe;
        break;
      }
      lo = probe;
    }
    while (hi - lo > 1u) {
      const uint32_t mid = lo + (hi - lo) / 2u;
      if ((ck[mid] >> GVIZ_SORT_SKIP_BITS) == key)
        lo = mid;
      else
        hi = mid;
    }
    end = hi;
  }
  const uint32_t len = end - start;
  if (len > k) {
    uint32_t slot = atomicAdd(&counts[1], 1u);
    deep[2 * slot] = start;
    deep[2 * slot + 1] = len;
  } else if (len >= 2) {
    // path bits covered by the sorted prefix of the composite key
    const int covered = 64 - GVIZ_SORT_SKIP_BITS - gbits;
    const uint64_t mask = covered >= 64 ? ~0ull : (~0ull << (64 - covered));
    for (uint32_t j = start; j < end; j++) {
      sHi[j] &= mask;
      sLo[j] = 0;
    }
  }
}

__device__ __forceinline__ bool key_less(uint64_t ah, uint64_t al, uint32_t av,
                                         uint64_t bh, uint64_t bl, uint32_t bv) {
  if (ah != bh) return ah < bh;
  if (al != bl) return al < bl;
  return av < bv;
}

// Bitonic sort of each deep run by (full path, vertex index) in shared memory.
__global__ __launch_bounds__(512) void k_sort_runs(
    uint64_t *sHi, uint64_t *sLo, uint32_t *idx, const uint32_t *__restrict__ deep,
    const uint32_t *__restrict__ counts, uint32_t *status) {
  extern __shared__ unsigned char smem[];
  uint64_t *kh = reinterpret_cast<uint64_t *>(smem);
  uint64_t *kl = kh + GVIZ_FIX_MAX;
  uint32_t *kv = reinterpret_cast<uint32_t *>(kl + GVIZ_FIX_MAX);
  const uint32_t nDeep = counts[1];
  for (uint32_t r = blockIdx.x; r < nDeep; r += gridDim.x) {
    const uint32_t start = deep[2 * r], len = deep[2 * r + 1];
    if (len > GVIZ_FIX_MAX) {
      int diff = 0;
      for (uint32_t j = threadIdx.x; j < len; j += blockDim.x) {
        if (sHi[start + j] != sHi[start] || sLo[start + j] != sLo[start]) diff = 1;
      }
      if (__syncthreads_or(diff) && threadIdx.x == 0)
        atomicOr(status, GVIZ_ST_DEEP_RUN);
      continue;
    }
    uint32_t P = 1;
    while (P < len) P <<= 1;
    for (uint32_t j = threadIdx.x; j < P; j += blockDim.x) {
      if (j < len) {
        kh[j] = sHi[start + j];
        kl[j] = sLo[start + j];
        kv[j] = idx[start + j];
      } else {
        kh[j] = ~0ull;
        kl[j] = ~0ull;
        kv[j] = ~0u;
      }
    }
    __syncthreads();
    for (uint32_t size = 2; size <= P; size <<= 1) {
      for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
        for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
          uint32_t j = i ^ stride;
          if (j > i) {
            bool asc = (i & size) == 0;
            bool gt = key_less(kh[j], kl[j], kv[j], kh[i], kl[i], kv[i]);
            if (gt == asc) {
              uint64_t t64 = kh[i];
              kh[i] = kh[j];
              kh[j] = t64;
              t64 = kl[i];
              kl[i] = kl[j];
              kl[j] = t64;
              uint32_t t32 = kv[i];
              kv[i] = kv[j];
              kv[j] = t32;
            }
          }
        }
        __syncthreads();
      }
    }
    for (uint32_t j = threadIdx.x; j < len; j += blockDim.x) {
      sHi[start + j] = kh[j];
      sLo[start + j] = kl[j];
      idx[start + j] = kv[j];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// buckets (identical full paths) and the binary radix tree
// ---------------------------------------------------------------------------

__global__ __launch_bounds__(kThreads) void k_bucket_flags(
    const uint64_t *__restrict__ sHi, const uint64_t *__restrict__ sLo,
    const uint32_t *__restrict__ idx, const uint32_t *__restrict__ gid,
    uint32_t *flag, uint32_t V) {
  uint32_t s = blockIdx.x * kThreads + threadIdx.x;
  if (s >= V) return;
  uint32_t f = 1;
  if (s > 0) {
    f = (sHi[s] != sHi[s - 1] || sLo[s] != sLo[s - 1]) ? 1u : 0u;
    if (!f && gid) f = gid[idx[s]] != gid[idx[s - 1]];
  }
  flag[s] = f;
}

__global__ __launch_bounds__(kThreads) void k_bucket_fill(
    const uint32_t *__restrict__ flag, const uint32_t *__restrict__ scan,
    const uint64_t *__restrict__ sHi, const uint64_t *__restrict__ sLo,
    const uint32_t *__restrict__ idx, const uint32_t *__restrict__ gid,
    uint32_t *bStart, uint64_t *bHi, uint64_t *bLo, uint32_t *bGid,
    uint2 *upLeaf, uint32_t V) {
  uint32_t s = blockIdx.x * kThreads + threadIdx.x;
  if (s >= V || !flag[s]) return;
  uint32_t b = scan[s];
  bStart[b] = s;
  bHi[b] = sHi[s];
  bLo[b] = sLo[s];
  bGid[b] = gid ? gid[idx[s]] : 0u;
  upLeaf[b] = make_uint2(GVIZ_NONE, 0u);
}

// Common-prefix length in bits of the composite keys (graph id:32,
// path:128) of buckets a and b; -1 outside [0, U). Keys of buckets
// [T0, T0 + kKarrasTile) come from the block's shared-memory copy; bGid is
// null for a single graph (every graph id is 0).
constexpr int kKarrasTile = 3 * kThreads;

struct KarrasKeys {
  const uint64_t *bHi, *bLo;
  const uint32_t *bGid;
  const uint64_t *sHi, *sLo;  // shared copies of [T0, T0 + kKarrasTile)
  int T0, U;
  __device__ __forceinline__ uint64_t hi(int b) const {
    return (unsigned)(b - T0) < (unsigned)kKarrasTile ? sHi[b - T0] : bHi[b];
  }
  __device__ __forceinline__ uint64_t lo(int b) const {
    return (unsigned)(b - T0) < (unsigned)kKarrasTile ? sLo[b - T0] : bLo[b];
  }
};

__device__ __forceinline__ int bdelta(int a, int b, const KarrasKeys &k) {
  if (b < 0 || b >= k.U) return -1;
  if (k.bGid) {
    uint32_t gx = k.bGid[a] ^ k.bGid[b];
    if (gx) return __clz(gx);
  }
  uint64_t x = k.hi(a) ^ k.hi(b);
  if (x) return 32 + __clzll(x);
  x = k.lo(a) ^ k.lo(b);
  if (x) return 96 + __clzll(x);
  return 160;
}

// Karras, "Maximizing parallelism in the construction of BVHs, octrees and
// k-d trees" (HPG 2012), algorithm of section 4 over unique bucket keys.
// Block j finds nodes [256 j, 256 j + 256); the keys of the 256 buckets on
// either side are staged in shared memory first, where most of the
// searches stay.
__global__ __launch_bounds__(kThreads) void k_karras(
    const uint64_t *__restrict__ bHi, const uint64_t *__restrict__ bLo,
    const uint32_t *__restrict__ bGid, const uint32_t *__restrict__ counts,
    uint32_t *nLeft, uint32_t *nRight, uint32_t *nFirst, uint32_t *nLast,
    int32_t *nDelta, uint2 *upInt, uint2 *upLeaf) {
  __shared__ uint64_t sHi[kKarrasTile], sLo[kKarrasTile];
  const int U = (int)counts[2];
  const int B0 = (int)(blockIdx.x * kThreads);
  if (B0 >= U - 1) return;
  KarrasKeys k{bHi, bLo, bGid, sHi, sLo, B0 - kThreads, U};
  for (int j = threadIdx.x; j < kKarrasTile; j += kThreads) {
    const int b = k.T0 + j;
    if (b >= 0 && b < U) {
      sHi[j] = bHi[b];
      sLo[j] = bLo[b];
    }
  }
  __syncthreads();
  const int i = B0 + threadIdx.x;
  if (i >= U - 1) return;
  const int dir = (bdelta(i, i + 1, k) - bdelta(i, i - 1, k)) >= 0 ? 1 : -1;
  const int dmin = bdelta(i, i - dir, k);
  int lmax = 2;
  while (bdelta(i, i + lmax * dir, k) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (bdelta(i, i + (l + t) * dir, k) > dmin) l += t;
  const int j = i + l * dir;
  const int dnode = bdelta(i, j, k);
  int s = 0;
  int div = 2;
  int t;
  do {
    t = (l + div - 1) / div;
    if (bdelta(i, i + (s + t) * dir, k) > dnode) s += t;
    div <<= 1;
  } while (t > 1);
  const int gamma = i + s * dir + min(dir, 0);
  const int first = min(i, j), last = max(i, j);
  uint32_t left, right;
  if (first == gamma) {
    left = (uint32_t)gamma | GVIZ_LEAF_BIT;
    upLeaf[gamma].x = (uint32_t)i;
  } else {
    left = (uint32_t)gamma;
    upInt[gamma].x = (uint32_t)i;
  }
  if (last == gamma + 1) {
    right = (uint32_t)(gamma + 1) | GVIZ_LEAF_BIT;
    upLeaf[gamma + 1].x = (uint32_t)i;
  } else {
    right = (uint32_t)(gamma + 1);
    upInt[gamma + 1].x = (uint32_t)i;
  }
  nLeft[i] = left;
  nRight[i] = right;
  nFirst[i] = (uint32_t)first;
  nLast[i] = (uint32_t)last;
  nDelta[i] = dnode;
  if (i == 0) upInt[0].x = GVIZ_NONE;
}

struct BU {
  const uint32_t *idx, *bStart, *bGid, *counts, *nLeft, *nRight, *nFirst, *nLast;
  const int32_t *nDelta;
  const double *mass;
  const double2 *pos;
  uint2 *upInt, *upLeaf;
  uint32_t *nCounter;
  double *bM, *bSX, *bSY, *nM, *nSX, *nSY;
  uint32_t *bCnt, *bT, *nCnt, *nT, *nFlag, *rootNode, *rootT, *status;
  // second central moments {Qxx, Qxy, Qyy, -}, or null: summed and shifted
  // in FP64, stored in FP32 (they only feed FP32 features)
  float4 *bQ, *nQ;
  // nodes spanning blocks whose children are both summed when k_bottom_up
  // ends (counts[4] of them)
  uint32_t *ready;
  uint32_t V, k;
};

// second central moments of a child about its own centre of mass
__device__ __forceinline__ float4 child_q(const BU &a, uint32_t c) {
  return (c & GVIZ_LEAF_BIT) ? a.bQ[c & ~GVIZ_LEAF_BIT] : a.nQ[c];
}

// parallel-axis shift of a child's moments to the parent's centre of mass
// (px, py): M_c (c_c - p)^2 = (S_c - M_c p)^2 / M_c, the difference in FP64,
// the rest in FP32 like the stored moments
__device__ __forceinline__ void add_shifted(float4 &q, const float4 qc, double M, double SX,
                                            double SY, double px, double py) {
  q.x += qc.x;
  q.y += qc.y;
  q.z += qc.z;
  if (M > 1e-9 || M < -1e-9) {
    const float tx = (float)(SX - M * px), ty = (float)(SY - M * py);
    const float im = 1.0f / (float)M;
    q.x += tx * tx * im;
    q.y += tx * ty * im;
    q.z += ty * ty * im;
  }
}

__device__ __forceinline__ void child_vals(const BU &a, uint32_t c, double &M,
                                           double &SX, double &SY,
                                           uint32_t &cnt, uint32_t &T) {
  // plain loads: the acquire on the arrival counter (block or device scope)
  // makes the sibling's stores visible
  if (c & GVIZ_LEAF_BIT) {
    uint32_t b = c & ~GVIZ_LEAF_BIT;
    M = a.bM[b];
    SX = a.bSX[b];
    SY = a.bSY[b];
    cnt = a.bCnt[b];
    T = a.bT[b];
  } else {
    M = a.nM[c];
    SX = a.nSX[c];
    SY = a.nSY[c];
    cnt = a.nCnt[c];
    T = a.nT[c];
  }
}

__device__ __forceinline__ uint2 *up_of(const BU &a, uint32_t c) {
  return (c & GVIZ_LEAF_BIT) ? a.upLeaf + (c & ~GVIZ_LEAF_BIT) : a.upInt + c;
}

// Node p from its children l, r (left first: fixed order, deterministic
// sums): mass, mass-weighted position sums, point count, subtree size in
// emitted records, the absorbed (p shares its quadtree level with its parent
// pp) and collapsed (a capacity leaf) flags and its children's preorder link
// weights; with kQ the second moments about p's centre of mass.
template <bool kQ>
__device__ __forceinline__ void combine(const BU &a, uint32_t p, int dp, uint32_t pp, int dpp,
                                        uint32_t l, uint32_t r, double Ml, double SXl,
                                        double SYl, uint32_t cl, uint32_t Tl, float4 ql,
                                        double Mr, double SXr, double SYr, uint32_t cr,
                                        uint32_t Tr, float4 qr, double &M, double &SX,
                                        double &SY, uint32_t &cnt, uint32_t &T,
                                        float4 &q) {
  M = Ml + Mr;
  SX = SXl + SXr;
  SY = SYl + SYr;
  cnt = cl + cr;
  const bool absorbed = pp != GVIZ_NONE && dpp >= 32 && ((dp - 32) >> 1) == ((dpp - 32) >> 1);
  const bool collapsed = !absorbed && cnt <= a.k;
  T = absorbed ? Tl + Tr : (collapsed ? 1u + cnt : 1u + Tl + Tr);
  if (kQ) {
    double px = 0.0, py = 0.0;
    if (M > 1e-9 || M < -1e-9) {
      const double im = __drcp_rn(M);  // one reciprocal on the serial climb
      px = SX * im;
      py = SY * im;
    }
    q = make_float4(0.f, 0.f, 0.f, 0.f);
    add_shifted(q, ql, Ml, SXl, SYl, px, py);
    add_shifted(q, qr, Mr, SXr, SYr, px, py);
    a.nQ[p] = q;
  }
  a.nM[p] = M;
  a.nSX[p] = SX;
  a.nSY[p] = SY;
  a.nCnt[p] = cnt;
  a.nT[p] = T;
  a.nFlag[p] = (absorbed ? 1u : 0u) | (collapsed ? 2u : 0u);
  const uint32_t base = absorbed ? 0u : 1u;
  const uint32_t dead = collapsed ? 0x80000000u : 0u;
  up_of(a, l)->y = base | dead;
  up_of(a, r)->y = (base + Tl) | dead;
}

// Per-block shared state of k_bottom_up: the sums of the block's buckets
// [B0, B1) (slot b - B0), the sums of its in-block internal nodes (slot
// p - B0; a Karras node is one end of its own range, so an internal node
// whose bucket range lies in [B0, B1) has its index there too) and the shape
// of the internal nodes [B0, B1), loaded once and coalesced.
template <bool kQ>
struct BUShared {
  uint32_t arrive[kThreads];
  double lM[kThreads], lSX[kThreads], lSY[kThreads];
  double iM[kThreads], iSX[kThreads], iSY[kThreads];
  uint32_t lCnt[kThreads], lT[kThreads], iCnt[kThreads], iT[kThreads];
  uint32_t left[kThreads], right[kThreads], first[kThreads], last[kThreads], up[kThreads];
  int32_t delta[kThreads];
  float4 lQ[kQ ? kThreads : 1], iQ[kQ ? kThreads : 1];
};

// Sums per bucket, then each thread climbs; the second child to arrive at a
// node combines both (left first: fixed order, deterministic sums). A node
// whose buckets all belong to this block has both children summed by
// threads of this block: its arrivals meet in shared memory with block-scope
// ordering and its children's sums are read from shared memory. A climb
// stops at the first node spanning blocks: its arrivals use a device-scope
// counter, and the second one lists the node for k_bottom_up_top. (A block
// that carried its climbs to the root stayed resident for ~20 device-scope
// steps, and the kernel ran in several such waves.) Every node's sums also
// go to global memory (k_emit reads them).
template <bool kQ>
__global__ __launch_bounds__(kThreads) void k_bottom_up(BU a) {
  __shared__ BUShared<kQ> s;
  const uint32_t U = a.counts[2];
  const uint32_t B0 = blockIdx.x * kThreads;
  const uint32_t B1 = min(B0 + kThreads, U);
  const uint32_t tid = threadIdx.x;
  s.arrive[tid] = 0u;
  if (B0 + tid + 1 < U) {  // internal nodes are [0, U - 1)
    const uint32_t p = B0 + tid;
    s.left[tid] = a.nLeft[p];
    s.right[tid] = a.nRight[p];
    s.first[tid] = a.nFirst[p];
    s.last[tid] = a.nLast[p];
    s.up[tid] = a.upInt[p].x;
    s.delta[tid] = a.nDelta[p];
  }
  __syncthreads();
  const uint32_t b = B0 + tid;
  if (b >= U) return;
  const uint32_t start = a.bStart[b];
  const uint32_t end = (b + 1 < U) ? a.bStart[b + 1] : a.V;
  double M = 0.0, SX = 0.0, SY = 0.0;
  for (uint32_t j = start; j < end; j++) {
    uint32_t i = a.idx[j];
    double m = a.mass[i];
    double2 p = a.pos[i];
    M += m;
    SX += m * p.x;
    SY += m * p.y;
  }
  uint32_t cnt = end - start;
  uint32_t T = cnt == 1 ? 1u : 1u + cnt;
  if (kQ) {
    double cx = 0.0, cy = 0.0;
    if (M > 1e-9 || M < -1e-9) {
      cx = SX / M;
      cy = SY / M;
    }
    // a single point has no second moments about itself: the bucket's own
    // pass over its points runs only for two or more
    double4 q = make_double4(0.0, 0.0, 0.0, 0.0);
    for (uint32_t j = start; cnt > 1u && j < end; j++) {
      const uint32_t i = a.idx[j];
      const double m = a.mass[i];
      const double2 p = a.pos[i];
      const double dx = p.x - cx, dy = p.y - cy;
      q.x += m * dx * dx;
      q.y += m * dx * dy;
      q.z += m * dy * dy;
    }
    const float4 fq = make_float4((float)q.x, (float)q.y, (float)q.z, 0.f);
    a.bQ[b] = fq;
    s.lQ[tid] = fq;
  }
  a.bM[b] = M;
  a.bSX[b] = SX;
  a.bSY[b] = SY;
  a.bCnt[b] = cnt;
  a.bT[b] = T;
  s.lM[tid] = M;
  s.lSX[tid] = SX;
  s.lSY[tid] = SY;
  s.lCnt[tid] = cnt;
  s.lT[tid] = T;
  const uint32_t g = a.bGid[b];
  uint32_t x = b | GVIZ_LEAF_BIT;
  uint32_t p = a.upLeaf[b].x;
  for (int guard = 0;; guard++) {
    if (guard > GVIZ_MAX_CLIMB) {
      atomicOr(a.status, GVIZ_ST_TREE);
      return;
    }
    const bool pin = p >= B0 && p < B1;  // false for GVIZ_NONE
    const int dp = p == GVIZ_NONE ? 0 : (pin ? s.delta[p - B0] : a.nDelta[p]);
    if (p == GVIZ_NONE || dp < 32) {
      a.rootNode[g] = x;
      a.rootT[g] = T;
      *up_of(a, x) = make_uint2(GVIZ_NONE, 0u);
      return;
    }
    if (!pin || s.first[p - B0] < B0 || s.last[p - B0] >= B1) {
      // a node spanning blocks: k_bottom_up_top sums it once both children
      // are summed
      cuda::atomic_ref<uint32_t, cuda::thread_scope_device> arrivals(a.nCounter[p]);
      if (arrivals.fetch_add(1u, cuda::memory_order_acq_rel) == 0u) return;
      a.nCounter[p] = 0u;
      a.ready[atomicAdd(const_cast<uint32_t *>(a.counts) + 4, 1u)] = p;
      return;
    }
    const uint32_t l = s.left[p - B0], r = s.right[p - B0], pp = s.up[p - B0];
    const int dpp = pp == GVIZ_NONE ? 0
                    : ((pp >= B0 && pp < B1) ? s.delta[pp - B0] : a.nDelta[pp]);
    // release this child's sums / acquire the sibling's: the second thread
    // to arrive combines both, reading them from shared memory (both
    // children lie in [B0, B1) and were summed by this block)
    cuda::atomic_ref<uint32_t, cuda::thread_scope_block> arrivals(s.arrive[p - B0]);
    if (arrivals.fetch_add(1u, cuda::memory_order_acq_rel) == 0u) return;
    double Ml, SXl, SYl, Mr, SXr, SYr;
    uint32_t cl, Tl, cr, Tr;
    float4 ql = make_float4(0.f, 0.f, 0.f, 0.f), qr = ql;
    if (l & GVIZ_LEAF_BIT) {
      const uint32_t c = (l & ~GVIZ_LEAF_BIT) - B0;
      Ml = s.lM[c], SXl = s.lSX[c], SYl = s.lSY[c], cl = s.lCnt[c], Tl = s.lT[c];
      if (kQ) ql = s.lQ[c];
    } else {
      const uint32_t c = l - B0;
      Ml = s.iM[c], SXl = s.iSX[c], SYl = s.iSY[c], cl = s.iCnt[c], Tl = s.iT[c];
      if (kQ) ql = s.iQ[c];
    }
    if (r & GVIZ_LEAF_BIT) {
      const uint32_t c = (r & ~GVIZ_LEAF_BIT) - B0;
      Mr = s.lM[c], SXr = s.lSX[c], SYr = s.lSY[c], cr = s.lCnt[c], Tr = s.lT[c];
      if (kQ) qr = s.lQ[c];
    } else {
      const uint32_t c = r - B0;
      Mr = s.iM[c], SXr = s.iSX[c], SYr = s.iSY[c], cr = s.iCnt[c], Tr = s.iT[c];
      if (kQ) qr = s.iQ[c];
    }
    float4 q;
    combine<kQ>(a, p, dp, pp, dpp, l, r, Ml, SXl, SYl, cl, Tl, ql, Mr, SXr, SYr, cr, Tr, qr,
                M, SX, SY, cnt, T, q);
    const uint32_t c = p - B0;  // an in-block parent reads the sums from here
    s.iM[c] = M;
    s.iSX[c] = SX;
    s.iSY[c] = SY;
    s.iCnt[c] = cnt;
    s.iT[c] = T;
    if (kQ) s.iQ[c] = q;
    x = p;
    p = pp;
  }
}

// The nodes spanning blocks, from those whose children k_bottom_up summed:
// each thread takes one listed node, sums it from its children's sums and
// climbs on while it arrives second (device-scope counters; the first
// arrival may have come from k_bottom_up). The climb's critical path is the
// tree's depth above the blocks (~20 levels at 1M points), so each level
// issues the next level's shape loads before its arrival and reads only
// the sibling's sums (the climbing child's are in registers). A persistent
// grid: the list is short (~3 % of the nodes at 1M points).
template <bool kQ>
__global__ __launch_bounds__(kThreads) void k_bottom_up_top(BU a) {
  const uint32_t nReady = a.counts[4];
  for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < nReady;
       i += gridDim.x * kThreads) {
    uint32_t p = a.ready[i];
    // p's shape (p is no root sentinel: k_bottom_up checked it)
    int dp = a.nDelta[p];
    uint32_t l = a.nLeft[p], r = a.nRight[p], pp = a.upInt[p].x;
    int dpp = pp == GVIZ_NONE ? 0 : a.nDelta[pp];
    // the climbing child's sums (none for a listed node: both are read)
    uint32_t x = GVIZ_NONE, T = 0, cnt = 0;
    double M = 0.0, SX = 0.0, SY = 0.0;
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int guard = 0;; guard++) {
      if (guard > GVIZ_MAX_CLIMB) {
        atomicOr(a.status, GVIZ_ST_TREE);
        break;
      }
      // the next level's shape, fetched while this level waits
      const bool nextIn = pp != GVIZ_NONE && dpp >= 32;
      uint32_t l2 = 0, r2 = 0, ppp = GVIZ_NONE;
      if (nextIn) {
        l2 = a.nLeft[pp];
        r2 = a.nRight[pp];
        ppp = a.upInt[pp].x;
      }
      if (x != GVIZ_NONE) {
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> arrivals(a.nCounter[p]);
        if (arrivals.fetch_add(1u, cuda::memory_order_acq_rel) == 0u) break;
        a.nCounter[p] = 0u;
      }
      double Ml, SXl, SYl, Mr, SXr, SYr;
      uint32_t cl, Tl, cr, Tr;
      float4 ql = make_float4(0.f, 0.f, 0.f, 0.f), qr = ql;
      if (x == l) {
        Ml = M, SXl = SX, SYl = SY, cl = cnt, Tl = T, ql = q;
      } else {
        child_vals(a, l, Ml, SXl, SYl, cl, Tl);
        if (kQ) ql = child_q(a, l);
      }
      if (x == r) {
        Mr = M, SXr = SX, SYr = SY, cr = cnt, Tr = T, qr = q;
      } else {
        child_vals(a, r, Mr, SXr, SYr, cr, Tr);
        if (kQ) qr = child_q(a, r);
      }
      combine<kQ>(a, p, dp, pp, dpp, l, r, Ml, SXl, SYl, cl, Tl, ql, Mr, SXr, SYr, cr, Tr, qr,
                  M, SX, SY, cnt, T, q);
      x = p;
      if (!nextIn) {  // x is its graph's root
        const uint32_t g = a.bGid[a.nFirst[x]];
        a.rootNode[g] = x;
        a.rootT[g] = T;
        *up_of(a, x) = make_uint2(GVIZ_NONE, 0u);
        break;
      }
      p = pp;
      dp = dpp;
      l = l2;
      r = r2;
      pp = ppp;
      dpp = pp == GVIZ_NONE ? 0 : a.nDelta[pp];
    }
  }
}

// preorder position (without the graph base) and whether any ancestor is a
// collapsed (capacity) leaf
__device__ __forceinline__ void walk_up(uint2 u, const uint2 *__restrict__ upInt,
                                        uint32_t &pre, uint32_t &dead) {
  pre = 0;
  dead = 0;
  for (int guard = 0; u.x != GVIZ_NONE; guard++) {
    if (guard > GVIZ_MAX_CLIMB) {  // never expected: report as dead
      dead = 1;
      return;
    }
    pre += u.y & 0x7fffffffu;
    dead |= u.y >> 31;
    u = upInt[u.x];
  }
}

struct EM {
  const uint32_t *idx, *bStart, *bGid, *bCnt, *counts, *nFirst, *nLast, *nFlag,
      *nT, *nCnt, *graphBase, *nLeft, *nRight;
  const int32_t *nDelta;
  const uint2 *upInt, *upLeaf;
  const double *bM, *bSX, *bSY, *nM, *nSX, *nSY, *mass, *radius;
  const double2 *pos;
  const GraphRoot *roots;
  void *nodes;
  uint32_t *status;
  double theta;
  uint32_t V, k, maxNodes;
  int f64;
  // far-field side records (null unless requested)
  const float4 *bQ, *nQ;
  const uint64_t *bHi, *bLo;
  FarCell *cells;
  uint32_t *leafPre;
  uint32_t *cellCnt;  // per record: points below it, 1 for a point (null unless requested)
  uint4 *kids;        // per cell: its children's preorder slots (null unless requested)
  // per internal node (k_pre_top): its preorder position without the graph
  // base if it spans blocks of k_bottom_up, else kPreLocal
  const uint32_t *preTop;
};

__device__ __forceinline__ void put_count(const EM &a, uint32_t at, uint32_t c) {
  if (a.cellCnt && at < a.maxNodes) a.cellCnt[at] = c;
}

// the even bits of x (bit 2j -> bit j)
__device__ __forceinline__ uint64_t even_bits(uint64_t x) {
  x &= 0x5555555555555555ull;
  x = (x | (x >> 1)) & 0x3333333333333333ull;
  x = (x | (x >> 2)) & 0x0f0f0f0f0f0f0f0full;
  x = (x | (x >> 4)) & 0x00ff00ff00ff00ffull;
  x = (x | (x >> 8)) & 0x0000ffff0000ffffull;
  return (x | (x >> 16)) & 0x00000000ffffffffull;
}

// Geometric centre of the cell at `depth` on the path (hi, lo), in closed
// form: with E (S) the east (south) bits of the path's first `depth` levels
// read as an integer, the descent's steps of +-h0 / 2^d sum to
// cx = cx0 + h0 ((2E + 1) / 2^depth - 1), cy = cy0 - h0 ((2S + 1) / 2^depth - 1).
// (Only a model feature: FP64 rounding may differ from the step-by-step
// descent in the last bits.)
__device__ void cell_center(const GraphRoot &R, uint64_t hi, uint64_t lo,
                            int depth, double &cx, double &cy) {
  const uint64_t eh = even_bits(hi), sh = even_bits(hi >> 1);  // levels 1..32
  uint64_t E, S;
  if (depth <= 32) {
    E = depth > 0 ? eh >> (32 - depth) : 0ull;
    S = depth > 0 ? sh >> (32 - depth) : 0ull;
  } else {
    const uint64_t el = even_bits(lo), sl = even_bits(lo >> 1);  // levels 33..64
    E = (eh << (depth - 32)) | (el >> (64 - depth));
    S = (sh << (depth - 32)) | (sl >> (64 - depth));
  }
  const double ex = ldexp(2.0 * (double)E + 1.0, -depth) - 1.0;
  const double sy = ldexp(2.0 * (double)S + 1.0, -depth) - 1.0;
  cx = R.cx + R.h0 * ex;
  cy = R.cy - R.h0 * sy;
}

__device__ void put_far(const EM &a, uint32_t at, const GraphRoot &R,
                        uint32_t keyBucket, int depth, double h, float4 q,
                        double M, double SX, double SY, uint32_t s0,
                        uint32_t s1) {
  if (!a.cells || at >= a.maxNodes) return;
  const double im = (M > 1e-30 || M < -1e-30) ? 1.0 / M : 0.0;
  double comx = 0.0, comy = 0.0;
  if (M > 1e-9 || M < -1e-9) {
    comx = SX * im;
    comy = SY * im;
  }
  double gx, gy;
  cell_center(R, a.bHi[keyBucket], a.bLo[keyBucket], depth, gx, gy);
  const double ih = h > 0.0 ? 1.0 / h : 0.0;
  FarCell c;
  c.qa = (float)((q.x - q.z) * im);
  c.qb = (float)(2.0 * q.y * im);
  c.tr = (float)((q.x + q.z) * im);
  c.h = (float)h;
  c.ox = (float)((gx - comx) * ih);
  c.oy = (float)((gy - comy) * ih);
  c.s0 = s0;
  c.s1 = s1;
  a.cells[at] = c;
}

__device__ void put_cell(const EM &a, uint32_t at, double M, double SX,
                         double SY, double h, uint32_t next) {
  if (at >= a.maxNodes) {
    atomicOr(a.status, GVIZ_ST_TREE);
    return;
  }
  double cx = 0.0, cy = 0.0;
  if (M > 1e-9 || M < -1e-9) {
    cx = SX / M;
    cy = SY / M;
  }
  if (a.f64) {
    NodeD n;
    n.x = cx;
    n.y = cy;
    n.mass = M;
    n.size = h;
    n.next = (int32_t)next;
    n.info = -1;
    n.pad0 = n.pad1 = 0;
    reinterpret_cast<NodeD *>(a.nodes)[at] = n;
  } else {
    NodeF n;
    ds_split(cx, n.xh, n.xl);
    ds_split(cy, n.yh, n.yl);
    n.mass = (float)M;
    if (isinf(h)) {
      n.size = INFINITY;
    } else {
      double t = 2.0 * h / a.theta;
      n.size = (float)(t * t);
    }
    n.next = (int32_t)next;
    n.info = -1;
    reinterpret_cast<NodeF *>(a.nodes)[at] = n;
  }
}

// Point v's leaf record at preorder slot `at`, from its position, mass and
// radius.
__device__ void put_leaf_vals(const EM &a, uint32_t at, uint32_t v, double2 p, double m,
                              double r) {
  if (at >= a.maxNodes) {
    atomicOr(a.status, GVIZ_ST_TREE);
    return;
  }
  if (a.leafPre) a.leafPre[v] = at;
  put_count(a, at, 1u);  // every record has its point count: k_far_groups reads it first
  if (a.f64) {
    NodeD n;
    n.x = p.x;
    n.y = p.y;
    n.mass = m;
    n.size = r;
    n.next = (int32_t)(at + 1);
    n.info = (int32_t)v;
    n.pad0 = n.pad1 = 0;
    reinterpret_cast<NodeD *>(a.nodes)[at] = n;
  } else {
    NodeF n;
    ds_split(p.x, n.xh, n.xl);
    ds_split(p.y, n.yh, n.yl);
    n.mass = (float)m;
    n.size = (float)r;
    n.next = (int32_t)(at + 1);
    n.info = (int32_t)v;
    reinterpret_cast<NodeF *>(a.nodes)[at] = n;
  }
}

__device__ void put_leaf(const EM &a, uint32_t at, uint32_t v) {
  put_leaf_vals(a, at, v, a.pos[v], a.mass[v], a.radius[v]);
}

// Children of a cell for walks that expand several cells at once (a cell's
// first child is the next preorder slot, the others sit behind their elder
// siblings' subtrees): up to four preorder slots in quadrant order,
// GVIZ_NONE where a quadrant is empty; a cell whose children are a run of
// more than four points (a leaf bucket or a capacity leaf) stores
// {first slot, GVIZ_KIDS_RUN, count}.
__device__ __forceinline__ uint32_t link_weight(const EM &a, uint32_t c) {
  const uint2 u = (c & GVIZ_LEAF_BIT) ? a.upLeaf[c & ~GVIZ_LEAF_BIT] : a.upInt[c];
  return u.y & 0x7fffffffu;
}

__device__ void put_kids_run(const EM &a, uint32_t at, uint32_t c) {
  if (!a.kids || at >= a.maxNodes) return;
  a.kids[at] = c <= 4u ? make_uint4(at + 1u, c > 1u ? at + 2u : GVIZ_NONE,
                                    c > 2u ? at + 3u : GVIZ_NONE, c > 3u ? at + 4u : GVIZ_NONE)
                       : make_uint4(at + 1u, GVIZ_KIDS_RUN, c, 0u);
}

// A quadtree node p: its binary children, or their children where a child
// was absorbed into p's level (two path bits per quadtree level), each at p's
// slot plus the weights of the links down to it.
__device__ void put_kids_quad(const EM &a, uint32_t at, uint32_t p) {
  if (!a.kids || at >= a.maxNodes) return;
  uint32_t out[4] = {GVIZ_NONE, GVIZ_NONE, GVIZ_NONE, GVIZ_NONE};
  int n = 0;
  const uint32_t ch[2] = {a.nLeft[p], a.nRight[p]};
  for (int i = 0; i < 2; i++) {
    const uint32_t c = ch[i];
    const uint32_t wc = at + link_weight(a, c);
    if (!(c & GVIZ_LEAF_BIT) && (a.nFlag[c] & 1u)) {
      const uint32_t g0 = a.nLeft[c], g1 = a.nRight[c];
      if (n < 4) out[n++] = wc + link_weight(a, g0);
      if (n < 4) out[n++] = wc + link_weight(a, g1);
    } else if (n < 4) {
      out[n++] = wc;
    }
  }
  a.kids[at] = make_uint4(out[0], out[1], out[2], out[3]);
}

// depth of the nearest quadtree ancestor of a node whose binary parent is p
__device__ __forceinline__ int quad_parent_depth(const EM &a, uint32_t p) {
  if (p != GVIZ_NONE && (a.nFlag[p] & 1u)) p = a.upInt[p].x;
  return p == GVIZ_NONE ? -1 : ((a.nDelta[p] - 32) >> 1);
}

// The records of internal node p (a quadtree cell or a capacity leaf) at
// preorder position pre (without the graph base).
__device__ void emit_internal(const EM &a, uint32_t U, uint32_t p, uint32_t pre,
                              uint32_t fb, uint32_t g, double M, double SX, double SY,
                              uint32_t T) {
  const GraphRoot R = a.roots[g];
  if (a.nFlag[p] & 2u) {  // capacity leaf: wrapper + points in vertex order
    const uint32_t lb = a.nLast[p];
    const uint32_t s0 = a.bStart[fb];
    const uint32_t s1 = (lb + 1 < U) ? a.bStart[lb + 1] : a.V;
    put_cell(a, pre, M, SX, SY, INFINITY, pre + T);
    put_count(a, pre, s1 - s0);
    put_kids_run(a, pre, s1 - s0);
    uint32_t ids[GVIZ_MAX_NODES_PER_CELL];
    uint32_t c = s1 - s0;
    for (uint32_t j = 0; j < c; j++) {
      uint32_t v = a.idx[s0 + j];
      uint32_t q = j;
      while (q > 0 && ids[q - 1] > v) {
        ids[q] = ids[q - 1];
        q--;
      }
      ids[q] = v;
    }
    for (uint32_t j = 0; j < c; j++) put_leaf(a, pre + 1 + j, ids[j]);
    return;
  }
  const int q = (a.nDelta[p] - 32) >> 1;
  put_cell(a, pre, M, SX, SY, ldexp(R.h0, -q), pre + T);
  put_kids_quad(a, pre, p);
  if (a.cells) {
    const uint32_t lb = a.nLast[p];
    const uint32_t s0 = a.bStart[fb];
    const uint32_t s1 = (lb + 1 < U) ? a.bStart[lb + 1] : a.V;
    put_far(a, pre, R, fb, q, ldexp(R.h0, -q), a.nQ[p], M, SX, SY, s0, s1);
    put_count(a, pre, s1 - s0);
  }
}

// The records of bucket b (a point, or the points of one smallest cell
// behind a wrapper cell) at preorder position pre (without the graph base).
__device__ void emit_bucket(const EM &a, uint32_t U, uint32_t b, uint32_t pre, uint2 ub,
                            uint32_t g, uint32_t c, uint32_t s0) {
  const GraphRoot R = a.roots[g];
  const int qp = quad_parent_depth(a, ub.x);
  const bool testable = c > a.k && qp < R.D - 1;
  const double h = testable ? ldexp(R.h0, -(R.D - 1)) : (double)INFINITY;
  put_cell(a, pre, a.bM[b], a.bSX[b], a.bSY[b], h, pre + 1 + c);
  put_count(a, pre, c);
  put_kids_run(a, pre, c);
  if (a.cells && testable)
    put_far(a, pre, R, b, R.D - 1, h, a.bQ[b], a.bM[b], a.bSX[b], a.bSY[b], s0,
            s0 + c);
  for (uint32_t j = 0; j < c; j++) put_leaf(a, pre + 1 + j, a.idx[s0 + j]);
}

// A node's preorder position relative to its graph's base is the sum of the
// link weights up to the graph's root. k_pre_top stores it for every internal
// node spanning blocks (GVIZ_NONE below a capacity leaf) and kPreLocal for
// the others, so a walk up stops at the first ancestor spanning blocks.
constexpr uint32_t kPreLocal = 0xFFFFFFFEu;

__device__ __forceinline__ bool spans_blocks(uint32_t p, uint32_t first, uint32_t last,
                                             uint32_t U) {
  const uint32_t B0 = p & ~(uint32_t)(kThreads - 1);
  return first < B0 || last >= min(B0 + kThreads, U);
}

__global__ __launch_bounds__(kThreads) void k_pre_top(const EM a) {
  const uint32_t U = a.counts[2];
  const uint32_t p = blockIdx.x * kThreads + threadIdx.x;
  if (p + 1 >= U) return;  // internal nodes are [0, U - 1)
  if (a.nDelta[p] < 32 || !spans_blocks(p, a.nFirst[p], a.nLast[p], U)) {
    const_cast<uint32_t *>(a.preTop)[p] = kPreLocal;
    return;
  }
  uint32_t pre, dead;
  walk_up(a.upInt[p], a.upInt, pre, dead);  // its ancestors all span blocks
  const_cast<uint32_t *>(a.preTop)[p] = dead ? GVIZ_NONE : pre;
}

// Shared by the threads of one k_emit block: parent links and k_pre_top's
// entries of the internal nodes [C0, C0 + kEmitSpan).
constexpr uint32_t kEmitSpan = kThreads / 2;
struct EmitShared {
  uint2 up[kEmitSpan];
  uint32_t pre[kEmitSpan];
};

// Preorder position (without the graph base) of the node whose parent link
// is u: the link weights summed up to the first ancestor spanning blocks,
// whose own position k_pre_top wrote. dead: an ancestor is a capacity leaf.
__device__ __forceinline__ uint32_t emit_pre(const EM &a, const EmitShared &s, uint32_t C0,
                                             uint2 u, bool &dead) {
  uint32_t pre = 0;
  dead = false;
  for (int guard = 0; u.x != GVIZ_NONE; guard++) {
    if (guard > GVIZ_MAX_CLIMB || (u.y >> 31)) {  // the guard is never expected
      dead = true;
      return 0;
    }
    pre += u.y;
    const uint32_t x = u.x;
    const bool cached = x - C0 < kEmitSpan;
    const uint32_t t = cached ? s.pre[x - C0] : a.preTop[x];
    if (t != kPreLocal) {
      if (t == GVIZ_NONE) dead = true;
      return pre + t;
    }
    u = cached ? s.up[x - C0] : a.upInt[x];
  }
  return pre;
}

// Node and leaf records in preorder: block j emits internal nodes and
// buckets [C0, C0 + kEmitSpan), C0 = kEmitSpan j, one per thread.
__global__ __launch_bounds__(kThreads) void k_emit(EM a) {
  __shared__ EmitShared s;
  const uint32_t U = a.counts[2];
  const uint32_t nInt = U - 1;
  const uint32_t C0 = blockIdx.x * kEmitSpan;
  if (C0 >= U) return;
  const uint32_t i = threadIdx.x % kEmitSpan;
  const uint32_t t = C0 + i;
  if (threadIdx.x < kEmitSpan && t < nInt) {
    s.up[i] = a.upInt[t];
    s.pre[i] = a.preTop[t];
  }
  __syncthreads();
  // each record's inputs are loaded before the walk up, whose end (the
  // preorder position) only the stores need
  if (threadIdx.x < kEmitSpan) {
    if (t < nInt && a.nDelta[t] >= 32 && !(a.nFlag[t] & 1u)) {
      const uint32_t fb = a.nFirst[t];
      const double M = a.nM[t], SX = a.nSX[t], SY = a.nSY[t];
      const uint32_t T = a.nT[t];
      const uint32_t g = a.bGid[fb];
      const uint32_t base = a.graphBase[g];
      bool dead;
      uint32_t pre = s.pre[i];
      if (pre == kPreLocal)
        pre = emit_pre(a, s, C0, s.up[i], dead);
      else
        dead = pre == GVIZ_NONE;
      if (!dead) emit_internal(a, U, t, pre + base, fb, g, M, SX, SY, T);
    }
  } else if (t < U) {
    const uint2 ub = a.upLeaf[t];
    const uint32_t g = a.bGid[t], c = a.bCnt[t], s0 = a.bStart[t];
    const uint32_t base = a.graphBase[g];
    const uint32_t v = a.idx[s0];  // the point of a single-point bucket
    double2 pv = make_double2(0.0, 0.0);
    double mv = 0.0, rv = 0.0;
    if (c == 1) {
      pv = a.pos[v];
      mv = a.mass[v];
      rv = a.radius[v];
    }
    bool dead;
    const uint32_t pre = emit_pre(a, s, C0, ub, dead);
    if (dead) return;
    if (c == 1)
      put_leaf_vals(a, pre + base, v, pv, mv, rv);
    else
      emit_bucket(a, U, t, pre + base, ub, g, c, s0);
  }
}

// Target groups of the learned cell-group walk: every cell of at most
// kGroupMax points whose parent holds more (or a root of at most kGroupMax
// points) is one group. Consecutive such children of one parent are packed
// into one group while the sum stays <= kGroupMax and the rectangle of
// their quadrants holds no other child of the parent (NW+NE, SW+SE, NW+SW
// with NE empty, ...), so a group's bounding box never covers points that
// are not its own; a group is a preorder range [x, y). A cell of more than
// four children is a leaf bucket (all its points in one smallest cell): its
// points are cut into runs of kGroupMax. Thread t < total handles the
// children of node t; thread maxNodes + g the root of graph g. The order of
// the groups in the list does not matter: a group's forces depend only on
// the group.
constexpr uint32_t kGroupMax = 32;

struct GroupArgs {
  const NodeF *nodes;
  const uint4 *kids;
  const FarCell *cells;
  const uint32_t *cellCnt, *counts, *graphBase, *rootT;
  uint4 *groups;
  uint32_t *nGroups;
  uint32_t maxNodes, G, cap;
};

__device__ __forceinline__ int4 node_link(const NodeF *nodes, uint32_t j) {
  return __ldg(reinterpret_cast<const int4 *>(nodes + j) + 1);  // mass, size, next, info
}

// quadrant (NW 0, NE 1, SW 2, SE 3) of the point set of node j inside a
// cell centred at (cx, cy), from its centre of mass
__device__ __forceinline__ uint32_t child_quadrant(const NodeF *nodes, uint32_t j, double cx,
                                                   double cy) {
  const NodeF n = nodes[j];
  const double x = (double)n.xh + (double)n.xl, y = (double)n.yh + (double)n.yl;
  return (x >= cx ? 1u : 0u) | (y < cy ? 2u : 0u);
}

// Each thread finds its groups (at most four packs of a branching cell, a
// root, or the runs of a leaf bucket); one atomic per warp reserves the
// warp's slots.
__global__ __launch_bounds__(kThreads) void k_far_groups(GroupArgs a) {
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t total = min(a.counts[3], a.maxNodes);
  uint32_t px[4], py[4], pc[4];
  uint32_t np = 0;                 // packs held in px/py/pc
  uint32_t runX = 0, runEnd = 0;   // a leaf bucket's runs [runX, runEnd)
  if (t >= a.maxNodes) {
    const uint32_t g = t - a.maxNodes;
    if (g < a.G) {
      const uint32_t r = a.graphBase[g], T = a.rootT[g];
      if (T != 0 && r < total) {
        const uint32_t c = a.cellCnt[r];
        if (c <= kGroupMax) {
          px[0] = r;
          py[0] = min(r + T, total);
          pc[0] = c;
          np = 1;
        }
      }
    }
  } else if (t < total && a.cellCnt[t] > kGroupMax) {  // (a point's count is 1)
    const int4 l = node_link(a.nodes, t);
    {
      const uint32_t end = min(max((uint32_t)l.z, t + 1u), total);
      uint32_t chX[4], chY[4], chC[4], chQ[4];
      int nc = 0;
      // the children from the cell's child record (independent loads): a
      // run of more than four points is a leaf bucket
      const uint4 kd = a.kids[t];
      const bool bucket = kd.y == GVIZ_KIDS_RUN;
      if (!bucket) {
        const uint32_t kk[4] = {kd.x, kd.y, kd.z, kd.w};
#pragma unroll
        for (int i = 0; i < 4; i++)
          if (kk[i] > t && kk[i] < end) chX[nc++] = kk[i];
        for (int i = 0; i < nc; i++) {
          chY[i] = i + 1 < nc ? chX[i + 1] : end;
          chC[i] = a.cellCnt[chX[i]];
        }
      }
      if (bucket) {  // points of one smallest cell: runs of kGroupMax leaves
        runX = t + 1u;
        runEnd = end;
      } else {
        const NodeF pn = a.nodes[t];
        const FarCell pcell = a.cells[t];
        const double cx = (double)pn.xh + (double)pn.xl + (double)pcell.ox * (double)pcell.h;
        const double cy = (double)pn.yh + (double)pn.yl + (double)pcell.oy * (double)pcell.h;
        for (int i = 0; i < nc; i++) chQ[i] = child_quadrant(a.nodes, chX[i], cx, cy);
        int first = -1;
        uint32_t pcnt = 0, r0 = 0, r1 = 0, c0 = 0, c1 = 0;  // pack, its quadrant rectangle
        for (int i = 0; i <= nc; i++) {
          if (i < nc && chC[i] <= kGroupMax && first >= 0 && pcnt + chC[i] <= kGroupMax) {
            const uint32_t R0 = min(r0, chQ[i] >> 1), R1 = max(r1, chQ[i] >> 1);
            const uint32_t C0 = min(c0, chQ[i] & 1u), C1 = max(c1, chQ[i] & 1u);
            bool fits = true;
            for (int k = 0; k < nc; k++) {
              if (k >= first && k <= i) continue;
              const uint32_t r = chQ[k] >> 1, c = chQ[k] & 1u;
              if (r >= R0 && r <= R1 && c >= C0 && c <= C1) fits = false;
            }
            if (fits) {
              r0 = R0, r1 = R1, c0 = C0, c1 = C1;
              pcnt += chC[i];
              continue;
            }
          }
          if (first >= 0) {
            px[np] = chX[first];
            py[np] = chY[i - 1];
            pc[np] = pcnt;
            np++;
          }
          first = -1;
          if (i < nc && chC[i] <= kGroupMax) {  // a larger child is cut by its own thread
            first = i;
            pcnt = chC[i];
            r0 = r1 = chQ[i] >> 1;
            c0 = c1 = chQ[i] & 1u;
          }
        }
      }
    }
  }
  const uint32_t nRuns = (runEnd - runX + kGroupMax - 1u) / kGroupMax;
  const uint32_t mine = np + nRuns;
  uint32_t incl = mine;  // inclusive warp scan of the group counts
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  const uint32_t warpTotal = __shfl_sync(0xffffffffu, incl, 31);
  uint32_t base = 0;
  if (lane == 0 && warpTotal) base = atomicAdd(a.nGroups, warpTotal);
  base = __shfl_sync(0xffffffffu, base, 0) + incl - mine;
  for (uint32_t k = 0; k < np; k++)
    if (base + k < a.cap) a.groups[base + k] = make_uint4(px[k], py[k], pc[k], 0u);
  for (uint32_t k = 0; k < nRuns; k++) {
    const uint32_t x = runX + k * kGroupMax, y = min(x + kGroupMax, runEnd);
    if (base + np + k < a.cap) a.groups[base + np + k] = make_uint4(x, y, y - x, 0u);
  }
}

// Inspection: per vertex, the index of its target group.
__global__ __launch_bounds__(kThreads) void k_group_members(const NodeF *nodes,
                                                            const uint4 *groups,
                                                            const uint32_t *nGroups,
                                                            uint32_t cap, uint32_t *groupOf) {
  const uint32_t gi = blockIdx.x * kThreads + threadIdx.x;
  if (gi >= min(*nGroups, cap)) return;
  const uint4 G = groups[gi];
  for (uint32_t j = G.x; j < G.y; j++) {
    const int4 l = node_link(nodes, j);
    if (l.w >= 0) groupOf[l.w] = gi;
  }
}

// Inspection: per point, the depth of the reference leaf holding it.
__global__ __launch_bounds__(kThreads) void k_leaf_depth(EM a, int32_t *depthOut) {
  const uint32_t U = a.counts[2];
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  const uint32_t nInt = U - 1;
  if (t < nInt) {
    const uint32_t p = t;
    if (a.nDelta[p] < 32 || !(a.nFlag[p] & 2u) || (a.nFlag[p] & 1u)) return;
    uint32_t pre, dead;
    walk_up(a.upInt[p], a.upInt, pre, dead);
    if (dead) return;
    const int d = quad_parent_depth(a, a.upInt[p].x) + 1;
    const uint32_t fb = a.nFirst[p], lb = a.nLast[p];
    const uint32_t s0 = a.bStart[fb];
    const uint32_t s1 = (lb + 1 < U) ? a.bStart[lb + 1] : a.V;
    for (uint32_t s = s0; s < s1; s++) depthOut[a.idx[s]] = d;
    return;
  }
  const uint32_t b = t - nInt;
  if (t < nInt || b >= U) return;
  uint32_t pre, dead;
  walk_up(a.upLeaf[b], a.upInt, pre, dead);
  if (dead) return;
  const uint32_t c = a.bCnt[b];
  const GraphRoot R = a.roots[a.bGid[b]];
  const int d = c > a.k ? R.D : quad_parent_depth(a, a.upLeaf[b].x) + 1;
  const uint32_t s0 = a.bStart[b];
  for (uint32_t j = 0; j < c; j++) depthOut[a.idx[s0 + j]] = d;
}

EM make_em(gvizCudaForce *h) {
  EM a;
  a.idx = h->d_idx;
  a.bStart = h->d_bStart;
  a.bGid = h->d_bGid;
  a.bCnt = h->d_bCnt;
  a.counts = h->d_counts;
  a.nFirst = h->d_nFirst;
  a.nLast = h->d_nLast;
  a.nFlag = h->d_nFlag;
  a.nT = h->d_nT;
  a.nCnt = h->d_nCnt;
  a.graphBase = h->d_graphBase;
  a.nDelta = h->d_nDelta;
  a.upInt = h->d_upInt;
  a.upLeaf = h->d_upLeaf;
  a.bM = h->d_bM;
  a.bSX = h->d_bSX;
  a.bSY = h->d_bSY;
  a.nM = h->d_nM;
  a.nSX = h->d_nSX;
  a.nSY = h->d_nSY;
  a.mass = h->d_mass;
  a.radius = h->d_radius;
  a.pos = h->d_pos;
  a.roots = h->d_roots;
  a.nodes = h->d_nodes;
  a.status = h->d_status;
  a.maxNodes = (uint32_t)h->maxNodes;
  a.theta = h->params.theta;
  a.V = (uint32_t)h->V;
  a.k = h->params.nodesPerCell;
  a.f64 = h->params.precision == GVIZ_CUDA_FP64;
  a.bQ = h->farSide ? h->d_bQ : nullptr;
  a.nQ = h->farSide ? h->d_nQ : nullptr;
  a.bHi = h->d_bHi;
  a.bLo = h->d_bLo;
  a.cells = h->farSide ? h->d_cells : nullptr;
  a.leafPre = h->farSide ? h->d_leafPre : nullptr;
  a.cellCnt = (h->farSide && h->params.farCellGroups) ? h->d_cellCnt : nullptr;
  a.nLeft = h->d_nLeft;
  a.nRight = h->d_nRight;
  a.kids = a.f64 ? nullptr : h->d_kids;  // the FP32 walks expand cells by them
  a.preTop = nullptr;
  return a;
}

inline uint32_t blocks_for(size_t n) {
  return (uint32_t)((n + kThreads - 1) / kThreads);
}

}  // namespace

void enqueue_tree_build(gvizCudaForce *h) {
  const uint32_t V = (uint32_t)h->V;
  cudaStream_t st = h->stream;
  cudaMemsetAsync(h->d_counts, 0, 8 * sizeof(uint32_t), st);
  // graphs without vertices get no root: their subtree size must read 0
  cudaMemsetAsync(h->d_rootT, 0, h->G * sizeof(uint32_t), st);
  k_bbox_chunks<<<h->nChunks, kThreads, 0, st>>>(h->d_pos, h->d_chunkBegin,
                                                  h->d_chunkEnd, h->d_chunkBox,
                                                  h->d_status);
  k_graph_roots<<<(uint32_t)h->G, kThreads, 0, st>>>(
      h->d_chunkBox, h->d_gChunkBegin, h->d_gChunkEnd, h->d_roots,
      (uint32_t)h->G, h->d_status);
  k_keys<<<blocks_for(V), kThreads, 0, st>>>(h->d_pos, h->d_gid, h->d_roots,
                                             h->d_keyHi, h->d_keyLo, h->d_ck,
                                             h->d_idx, V, h->gbits);
  prof_mark(h, "tree_keys");
  radix_sort_pairs(h, h->d_ck, h->d_idx, h->d_ckAlt, h->d_idxAlt, V);
  k_gather_keys<<<blocks_for(V), kThreads, 0, st>>>(h->d_idx, h->d_keyHi, h->d_keyLo,
                                                    h->d_ck, h->d_sHi, h->d_sLo,
                                                    h->d_flag, V);
  k_runs<<<blocks_for(V), kThreads, 0, st>>>(h->d_ck, h->d_flag, h->d_counts, h->d_deepRuns,
                                             h->d_sHi, h->d_sLo, V, h->params.nodesPerCell,
                                             h->gbits);
  const size_t fixSmem = (size_t)GVIZ_FIX_MAX * 20;
  k_sort_runs<<<148, 512, fixSmem, st>>>(h->d_sHi, h->d_sLo, h->d_idx,
                                          h->d_deepRuns, h->d_counts,
                                          h->d_status);
  k_bucket_flags<<<blocks_for(V), kThreads, 0, st>>>(h->d_sHi, h->d_sLo,
                                                     h->d_idx, h->d_gid,
                                                     h->d_flag, V);
  scan_exclusive(h, h->d_flag, h->d_scan, V, h->d_counts + 2);
  k_bucket_fill<<<blocks_for(V), kThreads, 0, st>>>(
      h->d_flag, h->d_scan, h->d_sHi, h->d_sLo, h->d_idx, h->d_gid,
      h->d_bStart, h->d_bHi, h->d_bLo, h->d_bGid, h->d_upLeaf, V);
  prof_mark(h, "tree_buckets");
  k_karras<<<blocks_for(V), kThreads, 0, st>>>(
      h->d_bHi, h->d_bLo, h->G > 1 ? h->d_bGid : nullptr, h->d_counts, h->d_nLeft, h->d_nRight,
      h->d_nFirst, h->d_nLast, h->d_nDelta, h->d_upInt, h->d_upLeaf);
  BU bu;
  bu.idx = h->d_idx;
  bu.bStart = h->d_bStart;
  bu.bGid = h->d_bGid;
  bu.counts = h->d_counts;
  bu.nLeft = h->d_nLeft;
  bu.nRight = h->d_nRight;
  bu.nFirst = h->d_nFirst;
  bu.nLast = h->d_nLast;
  bu.nDelta = h->d_nDelta;
  bu.mass = h->d_mass;
  bu.pos = h->d_pos;
  bu.upInt = h->d_upInt;
  bu.upLeaf = h->d_upLeaf;
  bu.nCounter = h->d_nCounter;
  bu.bM = h->d_bM;
  bu.bSX = h->d_bSX;
  bu.bSY = h->d_bSY;
  bu.nM = h->d_nM;
  bu.nSX = h->d_nSX;
  bu.nSY = h->d_nSY;
  bu.bCnt = h->d_bCnt;
  bu.bT = h->d_bT;
  bu.nCnt = h->d_nCnt;
  bu.nT = h->d_nT;
  bu.nFlag = h->d_nFlag;
  bu.rootNode = h->d_rootNode;
  bu.rootT = h->d_rootT;
  bu.status = h->d_status;
  bu.V = V;
  bu.k = h->params.nodesPerCell;
  bu.bQ = h->farSide ? h->d_bQ : nullptr;
  bu.nQ = h->farSide ? h->d_nQ : nullptr;
  // free after the buckets: the list of nodes spanning blocks, and the
  // preorder positions of k_pre_top
  bu.ready = h->d_flag;
  // the nodes spanning blocks are a few percent of the buckets: one wave
  const uint32_t topBlocks = std::max(1u, std::min<uint32_t>(blocks_for(V), 148u * 4u));
  if (bu.bQ) {
    k_bottom_up<true><<<blocks_for(V), kThreads, 0, st>>>(bu);
    k_bottom_up_top<true><<<topBlocks, kThreads, 0, st>>>(bu);
  } else {
    k_bottom_up<false><<<blocks_for(V), kThreads, 0, st>>>(bu);
    k_bottom_up_top<false><<<topBlocks, kThreads, 0, st>>>(bu);
  }
  scan_exclusive(h, h->d_rootT, h->d_graphBase, h->G, h->d_counts + 3);
  EM em = make_em(h);
  em.preTop = h->d_scan;
  k_pre_top<<<blocks_for(V), kThreads, 0, st>>>(em);
  k_emit<<<(uint32_t)((V + kEmitSpan - 1) / kEmitSpan), kThreads, 0, st>>>(em);
  if (em.cellCnt && !em.f64) {
    GroupArgs ga;
    ga.nodes = reinterpret_cast<const NodeF *>(h->d_nodes);
    ga.kids = h->d_kids;
    ga.cells = h->d_cells;
    ga.cellCnt = h->d_cellCnt;
    ga.counts = h->d_counts;
    ga.graphBase = h->d_graphBase;
    ga.rootT = h->d_rootT;
    ga.groups = h->d_groups;
    ga.nGroups = h->d_groupCount;
    ga.maxNodes = (uint32_t)h->maxNodes;
    ga.G = (uint32_t)h->G;
    ga.cap = (uint32_t)(V ? V : 1);
    cudaMemsetAsync(h->d_groupCount, 0, sizeof(uint32_t), st);
    k_far_groups<<<blocks_for((size_t)h->maxNodes + h->G), kThreads, 0, st>>>(ga);
  }
  prof_mark(h, "tree_nodes");
}

void enqueue_tree_export(gvizCudaForce *h, int32_t *leafDepth) {
  EM em = make_em(h);
  k_leaf_depth<<<blocks_for(2 * h->V), kThreads, 0, h->stream>>>(em,
                                                                 leafDepth);
}

void enqueue_group_export(gvizCudaForce *h, uint32_t *groupOf) {
  const uint32_t cap = (uint32_t)(h->V ? h->V : 1);
  k_group_members<<<blocks_for(cap), kThreads, 0, h->stream>>>(
      reinterpret_cast<const NodeF *>(h->d_nodes), h->d_groups, h->d_groupCount, cap, groupOf);
}

void tree_set_smem_limits() {
  cudaFuncSetAttribute(k_sort_runs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       GVIZ_FIX_MAX * 20);
}

// Inspection: every cell of the compressed tree (branching nodes and
// multi-point leaves) at its preorder slot, with the reference node it
// stands for: depth, quadrant path, mass, centre of mass, point count.
namespace {

__device__ __forceinline__ uint64_t dmask_hi(int d) {
  return d <= 0 ? 0ull : (d >= 32 ? ~0ull : (~0ull << (64 - 2 * d)));
}
__device__ __forceinline__ uint64_t dmask_lo(int d) {
  return d <= 32 ? 0ull : (d >= 64 ? ~0ull : (~0ull << (128 - 2 * d)));
}

struct CellOut {
  int32_t *depth;
  uint64_t *hi, *lo, *cnt;
  double *mass, *cx, *cy;
  const uint64_t *bHi, *bLo;
};

__device__ void cell_out(const CellOut &o, uint32_t at, int d, uint32_t b,
                         double M, double SX, double SY, uint64_t c) {
  o.depth[at] = d;
  o.hi[at] = o.bHi[b] & dmask_hi(d);
  o.lo[at] = o.bLo[b] & dmask_lo(d);
  o.mass[at] = M;
  const bool ok = M > 1e-9 || M < -1e-9;
  o.cx[at] = ok ? SX / M : 0.0;
  o.cy[at] = ok ? SY / M : 0.0;
  o.cnt[at] = c;
}

__global__ __launch_bounds__(kThreads) void k_cell_dump(EM a, CellOut o) {
  const uint32_t U = a.counts[2];
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  const uint32_t nInt = U - 1;
  if (t < nInt) {
    const uint32_t p = t;
    if (a.nDelta[p] < 32 || (a.nFlag[p] & 1u)) return;
    uint32_t pre, dead;
    walk_up(a.upInt[p], a.upInt, pre, dead);
    if (dead) return;
    const uint32_t fb = a.nFirst[p];
    pre += a.graphBase[a.bGid[fb]];
    const int d = (a.nFlag[p] & 2u) ? quad_parent_depth(a, a.upInt[p].x) + 1
                                    : ((a.nDelta[p] - 32) >> 1);
    cell_out(o, pre, d, fb, a.nM[p], a.nSX[p], a.nSY[p], a.nCnt[p]);
    return;
  }
  const uint32_t b = t - nInt;
  if (t < nInt || b >= U) return;
  const uint32_t c = a.bCnt[b];
  if (c < 2) return;
  uint32_t pre, dead;
  walk_up(a.upLeaf[b], a.upInt, pre, dead);
  if (dead) return;
  const GraphRoot R = a.roots[a.bGid[b]];
  pre += a.graphBase[a.bGid[b]];
  const int d = c > a.k ? R.D : quad_parent_depth(a, a.upLeaf[b].x) + 1;
  cell_out(o, pre, d, b, a.bM[b], a.bSX[b], a.bSY[b], c);
}

}  // namespace

void enqueue_cell_dump(gvizCudaForce *h, int32_t *depth, uint64_t *hi,
                       uint64_t *lo, double *mass, double *cx, double *cy,
                       uint64_t *cnt) {
  EM em = make_em(h);
  CellOut o;
  o.depth = depth;
  o.hi = hi;
  o.lo = lo;
  o.cnt = cnt;
  o.mass = mass;
  o.cx = cx;
  o.cy = cy;
  o.bHi = h->d_bHi;
  o.bLo = h->d_bLo;
  k_cell_dump<<<blocks_for(2 * h->V), kThreads, 0, h->stream>>>(em, o);
}
