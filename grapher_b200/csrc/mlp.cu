// mlp.cu -- learned far-field correction: training-pair harvest, BF16
// tensor-core training (forward + backward + Adam) and batch inference.
//
// Training pairs come from this library's own tree: for sampled targets the
// walk is replayed with the learned opening rule (theta test, and a cell that
// contains the target is never accepted), and for every accepted cell the
// exact FP64 force of its points (the all-pairs formula of
// src/embedders/gvizForceEmbedder.c:104-115 restricted to the cell) is set
// against its monopole (the pseudo-body term of :63-69).
//
// Training: mini-batch gradient of the weighted mean squared error of the
// relative correction, one warp per block over 32-sample tiles; activations
// and gradients pass through shared memory in BF16, every GEMM is
// mma.sync m16n8k16 (BF16 in, FP32 accumulate); per-block gradient partials
// are summed in block order (deterministic), then Adam on FP32 masters.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "mlp.cuh"

// FP32 master layout (padded like MlpDev): w1t[64][16], b1[64], w2t[64][64],
// b2[64], w3t[8][64], b3[8]
#define MLP_PAD (MLP_HID * MLP_INP + MLP_HID + MLP_HID * MLP_HID + MLP_HID + MLP_OUTP * MLP_HID + MLP_OUTP)
#define OFF_W1 0
#define OFF_B1 (OFF_W1 + MLP_HID * MLP_INP)
#define OFF_W2 (OFF_B1 + MLP_HID)
#define OFF_B2 (OFF_W2 + MLP_HID * MLP_HID)
#define OFF_W3 (OFF_B2 + MLP_HID)
#define OFF_B3 (OFF_W3 + MLP_OUTP * MLP_HID)

struct gvizCudaMlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  float *d_w = nullptr;      // FP32 masters (MLP_PAD)
  float *d_m = nullptr, *d_v = nullptr;  // Adam moments
  MlpDev *d_dev = nullptr;   // BF16 copy used by the kernels
  float *d_grad = nullptr;   // per-block partials [blocks][MLP_PAD + 1]
  float *d_gsum = nullptr;   // reduced gradient + loss
  size_t gradBlocks = 0;
  uint64_t step = 0;
  bool tc = true;                // training kernels: tcgen05 (true) or mma.sync
  uint32_t *d_status = nullptr;  // set by a tcgen05 kernel that gave up waiting
  float *d_epochLoss = nullptr;  // per-epoch loss sums of a training run
  size_t epochCap = 0;
};

namespace {

constexpr int kTilesPerBlock = 4;

__device__ __forceinline__ bool is_real_param(int i) {
  if (i < OFF_B1) return (i % MLP_INP) < MLP_IN;          // w1t columns >= 10
  if (i >= OFF_W3 && i < OFF_B3) return (i - OFF_W3) / MLP_HID < MLP_OUT;
  if (i >= OFF_B3) return (i - OFF_B3) < MLP_OUT;
  return true;
}

__global__ void k_mlp_to_dev(const float *w, MlpDev *d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= MLP_PAD) return;
  const float x = is_real_param(i) ? w[i] : 0.f;
  if (i < OFF_B1) d->w1t[i] = __float2bfloat16_rn(x);
  else if (i < OFF_W2) d->b1[i - OFF_B1] = x;
  else if (i < OFF_B2) d->w2t[i - OFF_W2] = __float2bfloat16_rn(x);
  else if (i < OFF_W3) d->b2[i - OFF_B2] = x;
  else if (i < OFF_B3) d->w3t[i - OFF_W3] = __float2bfloat16_rn(x);
  else d->b3[i - OFF_B3] = x;
}

// Per-block shared layout of the training kernel (one warp per block).
struct TrainSmem {
  __nv_bfloat16 w1t[MLP_HID * MLP_INP];
  __nv_bfloat16 w2t[MLP_HID * MLP_HID];
  __nv_bfloat16 w3p[16 * MLP_HID];  // w3t padded to 16 rows (rows >= 8 zero)
  float b1[MLP_HID], b2[MLP_HID], b3[MLP_OUTP];
  __nv_bfloat16 x[32 * MLP_INP];
  __nv_bfloat16 h1[32 * MLP_HID];
  __nv_bfloat16 h2[32 * MLP_HID];
  __nv_bfloat16 dy[32 * 16];
  __nv_bfloat16 dh2[32 * MLP_HID];
  __nv_bfloat16 dh1[32 * MLP_HID];
  float g[MLP_PAD];  // gradient accumulator (same layout as the masters)
  float loss;
};

// Gradient of sum_s w_s |Y_s - T_s|^2 * scale over `n` samples (through the
// index list `order`, or in order when null).
__global__ __launch_bounds__(32) void k_mlp_grad(const float *__restrict__ w,
                                                 const float *__restrict__ X,
                                                 const float *__restrict__ T,
                                                 const float *__restrict__ Wt,
                                                 const uint32_t *__restrict__ order,
                                                 uint32_t n, float scale,
                                                 float *partial) {
  extern __shared__ __align__(16) unsigned char smraw[];
  TrainSmem &S = *reinterpret_cast<TrainSmem *>(smraw);
  const int l = threadIdx.x;
  const int g = l >> 2, t = l & 3;
  for (int i = l; i < MLP_HID * MLP_INP; i += 32)
    S.w1t[i] = __float2bfloat16_rn((i % MLP_INP) < MLP_IN ? w[OFF_W1 + i] : 0.f);
  for (int i = l; i < MLP_HID * MLP_HID; i += 32) S.w2t[i] = __float2bfloat16_rn(w[OFF_W2 + i]);
  for (int i = l; i < 16 * MLP_HID; i += 32)
    S.w3p[i] = __float2bfloat16_rn(i / MLP_HID < MLP_OUT ? w[OFF_W3 + i] : 0.f);
  for (int i = l; i < MLP_HID; i += 32) {
    S.b1[i] = w[OFF_B1 + i];
    S.b2[i] = w[OFF_B2 + i];
  }
  if (l < MLP_OUTP) S.b3[l] = l < MLP_OUT ? w[OFF_B3 + l] : 0.f;
  for (int i = l; i < MLP_PAD; i += 32) S.g[i] = 0.f;
  if (l == 0) S.loss = 0.f;
  __syncwarp();

  const uint32_t nTiles = (n + 31) / 32;
  const uint32_t tile0 = blockIdx.x * kTilesPerBlock;
  for (uint32_t tile = tile0; tile < min(tile0 + kTilesPerBlock, nTiles); tile++) {
    // ---- load 32 samples (row l) -------------------------------------
    const uint32_t sIdx = tile * 32 + l;
    const bool valid = sIdx < n;
    const uint32_t src = valid ? (order ? order[sIdx] : sIdx) : 0u;
    float tgt0 = 0.f, tgt1 = 0.f, wt = 0.f;
#pragma unroll
    for (int f = 0; f < MLP_INP; f++)
      S.x[l * MLP_INP + f] = __float2bfloat16_rn(valid && f < MLP_IN ? X[(size_t)src * MLP_IN + f] : 0.f);
    if (valid) {
      tgt0 = T[(size_t)src * 2];
      tgt1 = T[(size_t)src * 2 + 1];
      wt = Wt ? Wt[src] : 1.f;
    }
#pragma unroll
    for (int f = 0; f < 16; f++) S.dy[l * 16 + f] = __float2bfloat16_rn(0.f);
    __syncwarp();
    // ---- forward: layer 1 ------------------------------------------------
    for (int mt = 0; mt < 2; mt++) {
      uint32_t a[4];
      load_a(a, S.x, MLP_INP, mt * 16, 0);
      for (int nt = 0; nt < 8; nt++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        uint32_t b[2];
        load_b_nk(b, S.w1t, MLP_INP, 0, nt * 8);
        mma16816(c, a, b);
        const int col = nt * 8 + 2 * t, r0 = mt * 16 + g;
        S.h1[r0 * MLP_HID + col] = __float2bfloat16_rn(fmaxf(c[0] + S.b1[col], 0.f));
        S.h1[r0 * MLP_HID + col + 1] = __float2bfloat16_rn(fmaxf(c[1] + S.b1[col + 1], 0.f));
        S.h1[(r0 + 8) * MLP_HID + col] = __float2bfloat16_rn(fmaxf(c[2] + S.b1[col], 0.f));
        S.h1[(r0 + 8) * MLP_HID + col + 1] = __float2bfloat16_rn(fmaxf(c[3] + S.b1[col + 1], 0.f));
      }
    }
    __syncwarp();
    // ---- layer 2 ---------------------------------------------------------
    for (int mt = 0; mt < 2; mt++) {
      uint32_t a[4][4];
      for (int kt = 0; kt < 4; kt++) load_a(a[kt], S.h1, MLP_HID, mt * 16, kt * 16);
      for (int nt = 0; nt < 8; nt++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        for (int kt = 0; kt < 4; kt++) {
          uint32_t b[2];
          load_b_nk(b, S.w2t, MLP_HID, kt * 16, nt * 8);
          mma16816(c, a[kt], b);
        }
        const int col = nt * 8 + 2 * t, r0 = mt * 16 + g;
        S.h2[r0 * MLP_HID + col] = __float2bfloat16_rn(fmaxf(c[0] + S.b2[col], 0.f));
        S.h2[r0 * MLP_HID + col + 1] = __float2bfloat16_rn(fmaxf(c[1] + S.b2[col + 1], 0.f));
        S.h2[(r0 + 8) * MLP_HID + col] = __float2bfloat16_rn(fmaxf(c[2] + S.b2[col], 0.f));
        S.h2[(r0 + 8) * MLP_HID + col + 1] = __float2bfloat16_rn(fmaxf(c[3] + S.b2[col + 1], 0.f));
      }
    }
    __syncwarp();
    // ---- layer 3, loss and dY ---------------------------------------------
    __shared__ float yS[32 * 2];
    for (int mt = 0; mt < 2; mt++) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      for (int kt = 0; kt < 4; kt++) {
        uint32_t a[4], b[2];
        load_a(a, S.h2, MLP_HID, mt * 16, kt * 16);
        load_b_nk(b, S.w3p, MLP_HID, kt * 16, 0);
        mma16816(c, a, b);
      }
      if (t == 0) {
        const int r0 = mt * 16 + g;
        yS[r0 * 2] = c[0] + S.b3[0];
        yS[r0 * 2 + 1] = c[1] + S.b3[1];
        yS[(r0 + 8) * 2] = c[2] + S.b3[0];
        yS[(r0 + 8) * 2 + 1] = c[3] + S.b3[1];
      }
    }
    __syncwarp();
    {
      const float e0 = yS[l * 2] - tgt0, e1 = yS[l * 2 + 1] - tgt1;
      const float d0 = 2.f * scale * wt * e0, d1 = 2.f * scale * wt * e1;
      float ls = scale * wt * (e0 * e0 + e1 * e1);
      S.dy[l * 16 + 0] = __float2bfloat16_rn(d0);
      S.dy[l * 16 + 1] = __float2bfloat16_rn(d1);
      float s0 = d0, s1 = d1;
      for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        ls += __shfl_xor_sync(0xffffffffu, ls, o);
      }
      if (l == 0) {
        S.g[OFF_B3] += s0;
        S.g[OFF_B3 + 1] += s1;
        S.loss += ls;
      }
    }
    __syncwarp();
    // ---- dW3t[o][j] += sum_s dY[s][o] H2[s][j] ------------------------------
    for (int nt = 0; nt < 8; nt++) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      for (int kt = 0; kt < 2; kt++) {
        uint32_t a[4], b[2];
        load_a_t(a, S.dy, 16, 0, kt * 16);
        load_b_kn(b, S.h2, MLP_HID, kt * 16, nt * 8);
        mma16816(c, a, b);
      }
      const int col = nt * 8 + 2 * t;  // rows g (outputs 0..7); g+8 are padding
      S.g[OFF_W3 + g * MLP_HID + col] += c[0];
      S.g[OFF_W3 + g * MLP_HID + col + 1] += c[1];
    }
    // ---- dH2 = dY W3 (masked), db2 ------------------------------------------
    for (int mt = 0; mt < 2; mt++) {
      uint32_t a[4];
      load_a(a, S.dy, 16, mt * 16, 0);
      for (int nt = 0; nt < 8; nt++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        uint32_t b[2];
        load_b_kn(b, S.w3p, MLP_HID, 0, nt * 8);
        mma16816(c, a, b);
        const int col = nt * 8 + 2 * t, r0 = mt * 16 + g;
        const int i00 = r0 * MLP_HID + col, i10 = (r0 + 8) * MLP_HID + col;
        const float v00 = __bfloat162float(S.h2[i00]) > 0.f ? c[0] : 0.f;
        const float v01 = __bfloat162float(S.h2[i00 + 1]) > 0.f ? c[1] : 0.f;
        const float v10 = __bfloat162float(S.h2[i10]) > 0.f ? c[2] : 0.f;
        const float v11 = __bfloat162float(S.h2[i10 + 1]) > 0.f ? c[3] : 0.f;
        S.dh2[i00] = __float2bfloat16_rn(v00);
        S.dh2[i00 + 1] = __float2bfloat16_rn(v01);
        S.dh2[i10] = __float2bfloat16_rn(v10);
        S.dh2[i10 + 1] = __float2bfloat16_rn(v11);
        float s0 = v00 + v10, s1 = v01 + v11;
        for (int o = 4; o < 32; o <<= 1) {  // sum over g (lanes with equal t)
          s0 += __shfl_xor_sync(0xffffffffu, s0, o);
          s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        }
        if (g == 0) {
          S.g[OFF_B2 + col] += s0;
          S.g[OFF_B2 + col + 1] += s1;
        }
      }
    }
    __syncwarp();
    // ---- dW2t[j2][j1] += sum_s dH2[s][j2] H1[s][j1] --------------------------
    for (int mt = 0; mt < 4; mt++) {
      uint32_t a[2][4];
      for (int kt = 0; kt < 2; kt++) load_a_t(a[kt], S.dh2, MLP_HID, mt * 16, kt * 16);
      for (int nt = 0; nt < 8; nt++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        for (int kt = 0; kt < 2; kt++) {
          uint32_t b[2];
          load_b_kn(b, S.h1, MLP_HID, kt * 16, nt * 8);
          mma16816(c, a[kt], b);
        }
        const int col = nt * 8 + 2 * t, r0 = mt * 16 + g;
        S.g[OFF_W2 + r0 * MLP_HID + col] += c[0];
        S.g[OFF_W2 + r0 * MLP_HID + col + 1] += c[1];
        S.g[OFF_W2 + (r0 + 8) * MLP_HID + col] += c[2];
        S.g[OFF_W2 + (r0 + 8) * MLP_HID + col + 1] += c[3];
      }
    }
    // ---- dH1 = dH2 W2 (masked), db1 ------------------------------------------
    for (int mt = 0; mt < 2; mt++) {
      uint32_t a[4][4];
      for (int kt = 0; kt < 4; kt++) load_a(a[kt], S.dh2, MLP_HID, mt * 16, kt * 16);
      for (int nt = 0; nt < 8; nt++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        for (int kt = 0; kt < 4; kt++) {
          uint32_t b[2];
          load_b_kn(b, S.w2t, MLP_HID, kt * 16, nt * 8);
          mma16816(c, a[kt], b);
        }
        const int col = nt * 8 + 2 * t, r0 = mt * 16 + g;
        const int i00 = r0 * MLP_HID + col, i10 = (r0 + 8) * MLP_HID + col;
        const float v00 = __bfloat162float(S.h1[i00]) > 0.f ? c[0] : 0.f;
        const float v01 = __bfloat162float(S.h1[i00 + 1]) > 0.f ? c[1] : 0.f;
        const float v10 = __bfloat162float(S.h1[i10]) > 0.f ? c[2] : 0.f;
        const float v11 = __bfloat162float(S.h1[i10 + 1]) > 0.f ? c[3] : 0.f;
        S.dh1[i00] = __float2bfloat16_rn(v00);
        S.dh1[i00 + 1] = __float2bfloat16_rn(v01);
        S.dh1[i10] = __float2bfloat16_rn(v10);
        S.dh1[i10 + 1] = __float2bfloat16_rn(v11);
        float s0 = v00 + v10, s1 = v01 + v11;
        for (int o = 4; o < 32; o <<= 1) {
          s0 += __shfl_xor_sync(0xffffffffu, s0, o);
          s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        }
        if (g == 0) {
          S.g[OFF_B1 + col] += s0;
          S.g[OFF_B1 + col + 1] += s1;
        }
      }
    }
    __syncwarp();
    // ---- dW1t[j1][f] += sum_s dH1[s][j1] X[s][f] ------------------------------
    for (int mt = 0; mt < 4; mt++) {
      uint32_t a[2][4];
      for (int kt = 0; kt < 2; kt++) load_a_t(a[kt], S.dh1, MLP_HID, mt * 16, kt * 16);
      for (int nt = 0; nt < 2; nt++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        for (int kt = 0; kt < 2; kt++) {
          uint32_t b[2];
          load_b_kn(b, S.x, MLP_INP, kt * 16, nt * 8);
          mma16816(c, a[kt], b);
        }
        const int col = nt * 8 + 2 * t, r0 = mt * 16 + g;
        S.g[OFF_W1 + r0 * MLP_INP + col] += c[0];
        S.g[OFF_W1 + r0 * MLP_INP + col + 1] += c[1];
        S.g[OFF_W1 + (r0 + 8) * MLP_INP + col] += c[2];
        S.g[OFF_W1 + (r0 + 8) * MLP_INP + col + 1] += c[3];
      }
    }
    __syncwarp();
  }
  float *out = partial + (size_t)blockIdx.x * (MLP_PAD + 1);
  for (int i = l; i < MLP_PAD; i += 32) out[i] = S.g[i];
  if (l == 0) out[MLP_PAD] = S.loss;
}

// ---------------------------------------------------------------------------
// Training on the 5th-generation tensor cores (tcgen05): one CTA of 128
// threads takes tiles of 128 samples (thread r = sample r of the tile = row
// r of every M = 128 product); operands are staged in shared memory in the
// no-swizzle canonical layouts (core matrices of 8 rows x 16 bytes),
// accumulators live in tensor memory (TMEM), one thread issues the MMAs and
// their completion is signalled through an mbarrier.
//   D_act [128 x 64] (TMEM columns 0..63), reused by three products:
//     X H1-pre = X W1^T, H2-pre = H1 W2^T, dH1-pre = dH2 W2
//   D_grad [128 x 96] (columns 64..159), accumulated over the CTA's tiles:
//     [dH2 | dH1]^T [H1 | X | 1]: rows 0..63 give dW2 and (column 80) db2,
//     rows 64..127 give dW1 (columns 64..79) and db1 (column 80)
//   D_w3 [128 x 16] (columns 160..175): [H2 | 1 | 0]^T [dY | 0]: rows 0..63
//     give dW3^T, row 64 gives db3
// The shared-memory buffers serve two roles each: the MN-major operand
// [H1 | X | 1] (features x samples) is, read as K-major, the A operand of
// the first two products, and [dH2 | dH1] is, read as K-major, the A of the
// third. Layer 3 (64 -> 2) and dH2 = dY W3 run on the CUDA cores per thread.
// BF16 rounding happens where the mma.sync kernel (and the oracle) round.
// Every gradient entry is written by exactly one thread of the CTA.
// ---------------------------------------------------------------------------
constexpr int kTcThreads = 128;
constexpr int kTcTilesPerBlock = 1;
constexpr uint32_t kTcCols = 256;  // TMEM columns allocated (power of two >= 176)
constexpr uint32_t kTcColGrad = 64, kTcColW3 = 160;
constexpr uint32_t kTcSpin = 1u << 22;  // mbarrier polls before giving up

struct __align__(128) TcSmem {
  __nv_bfloat16 w1[64 * 16];     // K-major [n = hidden 1][k = input]
  __nv_bfloat16 w2[64 * 64];     // K-major [n = hidden 2][k = hidden 1]
  __nv_bfloat16 w2t[64 * 64];    // K-major [n = hidden 1][k = hidden 2]
  __nv_bfloat16 bst[96 * 128];   // MN-major [n: H1 0..63 | X 64..79 | 1 80][k = sample]
  __nv_bfloat16 ast[128 * 128];  // MN-major [m: dH2 0..63 | dH1 64..127][k = sample]
  __nv_bfloat16 a2[128 * 128];   // MN-major [m: H2 0..63 | 1 64][k = sample]
  __nv_bfloat16 b2[16 * 128];    // MN-major [n: dY 0..1][k = sample]
  float w3[2][64];               // layer 3, BF16-rounded
  float b1[64], b2v[64], b3[2];
  float red[4];
  unsigned long long bar;
  uint32_t tmem;
};

// byte offset of element (row r, column k) of a K-major operand whose
// 8-row groups are `sbo` bytes apart (K chunks of 8 elements 128 bytes apart)
__device__ __forceinline__ uint32_t kmaj_off(uint32_t r, uint32_t k, uint32_t sbo) {
  return (r & 7u) * 16u + (r >> 3) * sbo + (k >> 3) * 128u + (k & 7u) * 2u;
}
// byte offset of the 16-byte chunk holding elements n0..n0+7 (n0 % 8 == 0)
// of sample k in an MN-major operand whose 8-sample groups are `lbo` apart
__device__ __forceinline__ uint32_t mn_off(uint32_t n0, uint32_t k, uint32_t lbo) {
  return (k & 7u) * 16u + (n0 >> 3) * 128u + (k >> 3) * lbo;
}

// shared-memory matrix descriptor: start, leading (K-group) and stride
// (MN-group) byte offsets, version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(const void *p, uint32_t lbo, uint32_t sbo) {
  const uint32_t a = smem_u32(p);
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B
__host__ __device__ constexpr uint32_t tc_idesc(uint32_t M, uint32_t N, uint32_t aMN, uint32_t bMN) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (aMN << 15) | (bMN << 16) | ((N >> 3) << 17) |
         ((M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(const unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void proxy_fence() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Waits for the mbarrier phase with a bounded number of polls; false when
// it gave up.
__device__ __forceinline__ bool tc_wait(const unsigned long long *bar, uint32_t phase) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < kTcSpin; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tc_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float bfr(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// 8 BF16 values as one 16-byte chunk
__device__ __forceinline__ uint4 pack8(const float *v) {
  return make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]),
                    pack_bf16(v[6], v[7]));
}

__global__ __launch_bounds__(kTcThreads, 1) void k_mlp_grad_tc(
    const float *__restrict__ w, const float *__restrict__ X, const float *__restrict__ T,
    const float *__restrict__ Wt, const uint32_t *__restrict__ order, uint32_t n, float scale,
    float *partial, uint32_t *status) {
  extern __shared__ __align__(128) unsigned char tcraw[];
  TcSmem &S = *reinterpret_cast<TcSmem *>(tcraw);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  unsigned char *w1b = reinterpret_cast<unsigned char *>(S.w1);
  unsigned char *w2b = reinterpret_cast<unsigned char *>(S.w2);
  unsigned char *w2tb = reinterpret_cast<unsigned char *>(S.w2t);
  unsigned char *bstb = reinterpret_cast<unsigned char *>(S.bst);
  unsigned char *astb = reinterpret_cast<unsigned char *>(S.ast);
  unsigned char *a2b = reinterpret_cast<unsigned char *>(S.a2);
  unsigned char *b2b = reinterpret_cast<unsigned char *>(S.b2);
  // ---- weights and constant operand parts --------------------------------
  for (uint32_t i = tid; i < 64 * 16; i += kTcThreads) {
    const uint32_t r = i / 16, k = i % 16;
    *reinterpret_cast<__nv_bfloat16 *>(w1b + kmaj_off(r, k, 256)) =
        __float2bfloat16_rn(k < MLP_IN ? w[OFF_W1 + i] : 0.f);
  }
  for (uint32_t i = tid; i < 64 * 64; i += kTcThreads) {
    const uint32_t r = i / 64, k = i % 64;  // w2t master: [out r][in k]
    const __nv_bfloat16 v = __float2bfloat16_rn(w[OFF_W2 + i]);
    *reinterpret_cast<__nv_bfloat16 *>(w2b + kmaj_off(r, k, 1024)) = v;
    *reinterpret_cast<__nv_bfloat16 *>(w2tb + kmaj_off(k, r, 1024)) = v;
  }
  for (uint32_t i = tid; i < 2 * 64; i += kTcThreads) S.w3[i / 64][i % 64] = bfr(w[OFF_W3 + i]);
  for (uint32_t i = tid; i < 64; i += kTcThreads) {
    S.b1[i] = w[OFF_B1 + i];
    S.b2v[i] = w[OFF_B2 + i];
  }
  if (tid < 2) S.b3[tid] = w[OFF_B3 + tid];
  {
    // per sample: bst n 80..95 = [1, 0 ...], a2 m 64..127 = [1, 0 ...],
    // b2 n 8..15 = 0
    const float one[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float zero[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const uint32_t k = tid;
    *reinterpret_cast<uint4 *>(bstb + mn_off(80, k, 1536)) = pack8(one);
    *reinterpret_cast<uint4 *>(bstb + mn_off(88, k, 1536)) = pack8(zero);
    *reinterpret_cast<uint4 *>(a2b + mn_off(64, k, 2048)) = pack8(one);
    for (uint32_t n0 = 72; n0 < 128; n0 += 8)
      *reinterpret_cast<uint4 *>(a2b + mn_off(n0, k, 2048)) = pack8(zero);
    *reinterpret_cast<uint4 *>(b2b + mn_off(8, k, 256)) = pack8(zero);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&S.tmem)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = S.tmem;
  const uint32_t lane_base = tbase + ((warp * 32u) << 16);  // this warp's TMEM lanes
  const uint32_t idAct = tc_idesc(128, 64, 0, 0);
  const uint32_t idGrad = tc_idesc(128, 96, 1, 1);
  const uint32_t idW3 = tc_idesc(128, 16, 1, 1);
  uint32_t phase = 0;
  bool ok = true;
  float lossAcc = 0.f;
  const uint32_t nTiles = (n + kTcThreads - 1) / kTcThreads;
  const uint32_t t0 = blockIdx.x * kTcTilesPerBlock;
  const uint32_t t1 = min(t0 + kTcTilesPerBlock, nTiles);
  // issue (thread 0) a chain of MMAs after the block's shared-memory
  // writes, then wait for it everywhere
  // (ok stays block-uniform: a wait that gave up anywhere stops every thread)
  auto sync_issue_wait = [&](auto issue) {
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      issue();
      tc_commit(&S.bar);
    }
    const bool got = tc_wait(&S.bar, phase);
    phase ^= 1u;
    ok = __syncthreads_and(got ? 1 : 0) != 0;
    tc_fence_after();
  };
  for (uint32_t tile = t0; tile < t1 && ok; tile++) {
    const uint32_t sIdx = tile * kTcThreads + tid;
    const bool valid = sIdx < n;
    const uint32_t src = valid ? (order ? order[sIdx] : sIdx) : 0u;
    float x[16];
#pragma unroll
    for (int f = 0; f < 16; f++)
      x[f] = (valid && f < MLP_IN) ? X[(size_t)src * MLP_IN + f] : 0.f;
    const float tg0 = valid ? T[(size_t)src * 2] : 0.f, tg1 = valid ? T[(size_t)src * 2 + 1] : 0.f;
    const float wt = valid ? (Wt ? Wt[src] : 1.f) : 0.f;
    *reinterpret_cast<uint4 *>(bstb + mn_off(64, tid, 1536)) = pack8(x);
    *reinterpret_cast<uint4 *>(bstb + mn_off(72, tid, 1536)) = pack8(x + 8);
    // ---- layer 1: D_act = X W1^T (K = 16) -------------------------------
    sync_issue_wait([&] {
      tc_mma(tbase, tc_desc(bstb + 1024, 128, 1536), tc_desc(w1b, 128, 256), idAct, 0u);
    });
    if (!ok) break;
    float h1[64];
    uint32_t m1a = 0, m1b = 0;  // ReLU masks of layer 1 (bits 0..31, 32..63)
#pragma unroll
    for (int c = 0; c < 4; c++) tc_ld16(lane_base + 16 * c, h1 + 16 * c);
    tc_wait_ld();
#pragma unroll
    for (int j = 0; j < 64; j++) {
      const float v = fmaxf(h1[j] + S.b1[j], 0.f);
      h1[j] = v;
      if (v > 0.f) {
        if (j < 32) m1a |= 1u << j;
        else m1b |= 1u << (j - 32);
      }
    }
#pragma unroll
    for (int g = 0; g < 8; g++)
      *reinterpret_cast<uint4 *>(bstb + mn_off(8 * g, tid, 1536)) = pack8(h1 + 8 * g);
    // ---- layer 2: D_act = H1 W2^T (K = 64) -------------------------------
    sync_issue_wait([&] {
#pragma unroll
      for (uint32_t kk = 0; kk < 4; kk++)
        tc_mma(tbase, tc_desc(bstb + 256 * kk, 128, 1536), tc_desc(w2b + 256 * kk, 128, 1024),
               idAct, kk);
    });
    if (!ok) break;
    float h2[64];
#pragma unroll
    for (int c = 0; c < 4; c++) tc_ld16(lane_base + 16 * c, h2 + 16 * c);
    tc_wait_ld();
    float y0 = S.b3[0], y1 = S.b3[1];
#pragma unroll
    for (int j = 0; j < 64; j++) {
      h2[j] = bfr(fmaxf(h2[j] + S.b2v[j], 0.f));
      y0 += h2[j] * S.w3[0][j];
      y1 += h2[j] * S.w3[1][j];
    }
    // ---- layer 3 on the CUDA cores, loss and dY ----------------------------
    const float e0 = y0 - tg0, e1 = y1 - tg1;
    const float d0 = bfr(2.f * scale * wt * e0), d1 = bfr(2.f * scale * wt * e1);
    lossAcc += scale * wt * (e0 * e0 + e1 * e1);
    {
      const float dy[8] = {d0, d1, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      *reinterpret_cast<uint4 *>(b2b + mn_off(0, tid, 256)) = pack8(dy);
    }
    // dH2 = (dY W3) masked by H2 > 0, BF16
    float dh[64];
#pragma unroll
    for (int j = 0; j < 64; j++) dh[j] = h2[j] > 0.f ? d0 * S.w3[0][j] + d1 * S.w3[1][j] : 0.f;
#pragma unroll
    for (int g = 0; g < 8; g++) {
      *reinterpret_cast<uint4 *>(a2b + mn_off(8 * g, tid, 2048)) = pack8(h2 + 8 * g);
      *reinterpret_cast<uint4 *>(astb + mn_off(8 * g, tid, 2048)) = pack8(dh + 8 * g);
    }
    // ---- dH1 = dH2 W2 (K = 64) --------------------------------------------
    sync_issue_wait([&] {
#pragma unroll
      for (uint32_t kk = 0; kk < 4; kk++)
        tc_mma(tbase, tc_desc(astb + 256 * kk, 128, 2048), tc_desc(w2tb + 256 * kk, 128, 1024),
               idAct, kk);
    });
    if (!ok) break;
#pragma unroll
    for (int c = 0; c < 4; c++) tc_ld16(lane_base + 16 * c, dh + 16 * c);
    tc_wait_ld();
#pragma unroll
    for (int j = 0; j < 64; j++) {
      const bool on = j < 32 ? (m1a >> j) & 1u : (m1b >> (j - 32)) & 1u;
      dh[j] = on ? dh[j] : 0.f;
    }
#pragma unroll
    for (int g = 0; g < 8; g++)
      *reinterpret_cast<uint4 *>(astb + mn_off(64 + 8 * g, tid, 2048)) = pack8(dh + 8 * g);
    // ---- weight gradients, accumulated in TMEM over the CTA's tiles (K = 128)
    const uint32_t first = tile == t0 ? 1u : 0u;
    sync_issue_wait([&] {
#pragma unroll
      for (uint32_t kk = 0; kk < 8; kk++) {
        const uint32_t acc = (first && kk == 0) ? 0u : 1u;
        tc_mma(tbase + kTcColGrad, tc_desc(astb + 4096 * kk, 2048, 128),
               tc_desc(bstb + 3072 * kk, 1536, 128), idGrad, acc);
        tc_mma(tbase + kTcColW3, tc_desc(a2b + 4096 * kk, 2048, 128),
               tc_desc(b2b + 512 * kk, 256, 128), idW3, acc);
      }
    });
  }
  // ---- this CTA's gradient: row tid of D_grad and D_w3 ---------------------
  float *out = partial + (size_t)blockIdx.x * (MLP_PAD + 1);
  if (ok && t0 < t1) {
    float g[96], g3[16];
#pragma unroll
    for (int c = 0; c < 6; c++) tc_ld16(lane_base + kTcColGrad + 16 * c, g + 16 * c);
    tc_ld16(lane_base + kTcColW3, g3);
    tc_wait_ld();
    if (tid < 64) {
      for (int j = 0; j < 64; j++) out[OFF_W2 + tid * 64 + j] = g[j];
      out[OFF_B2 + tid] = g[80];
      out[OFF_W3 + tid] = g3[0];
      out[OFF_W3 + 64 + tid] = g3[1];
      for (int o = 2; o < MLP_OUTP; o++) out[OFF_W3 + o * 64 + tid] = 0.f;
    } else {
      const uint32_t r = tid - 64;
      for (int c = 0; c < MLP_INP; c++) out[OFF_W1 + r * MLP_INP + c] = g[64 + c];
      out[OFF_B1 + r] = g[80];
      if (tid == 64) {
        out[OFF_B3] = g3[0];
        out[OFF_B3 + 1] = g3[1];
        for (int o = 2; o < MLP_OUTP; o++) out[OFF_B3 + o] = 0.f;
      }
    }
  } else {
    for (uint32_t i = tid; i < MLP_PAD; i += kTcThreads) out[i] = 0.f;
  }
  // loss: the block's sum
  float l = lossAcc;
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((tid & 31u) == 0) S.red[warp] = l;
  tc_fence_before();
  __syncthreads();
  if (tid == 0) out[MLP_PAD] = ok ? (S.red[0] + S.red[1]) + (S.red[2] + S.red[3]) : NAN;
  if (!ok && tid == 0) atomicOr(status, 1u);
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase),
                 "r"(kTcCols)
                 : "memory");
  }
}

// Sum of the per-block partials in block order.
__global__ void k_mlp_reduce(const float *partial, uint32_t blocks, float *sum) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > MLP_PAD) return;
  float s = 0.f;
  for (uint32_t b = 0; b < blocks; b++) s += partial[(size_t)b * (MLP_PAD + 1) + i];
  sum[i] = s;
}

__global__ void k_mlp_adam(float *w, float *m, float *v, const float *grad,
                           float lr, float b1, float b2, float eps,
                           float c1, float c2, float *epochLoss, float batchSamples) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && epochLoss) *epochLoss += grad[MLP_PAD] * batchSamples;
  if (i >= MLP_PAD) return;
  if (!is_real_param(i)) {
    w[i] = 0.f;
    return;
  }
  const float gr = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * gr;
  const float vi = b2 * v[i] + (1.f - b2) * gr * gr;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Batch inference (tests, the error monitor): one warp per 32 rows.
__global__ __launch_bounds__(128) void k_mlp_infer(const MlpDev *__restrict__ Wg,
                                                   const float *__restrict__ X,
                                                   uint32_t n, float *Y) {
  __shared__ MlpSmem W;
  __shared__ __align__(16) __nv_bfloat16 xs[4][32 * MLP_XS];
  __shared__ float ys[4][32 * 2];
  mlp_stage(W, Wg);
  __syncthreads();
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const uint32_t row = (blockIdx.x * 4 + w) * 32 + l;
  for (int f = 0; f < MLP_INP; f++)
    xs[w][l * MLP_XS + f] = __float2bfloat16_rn(row < n && f < MLP_IN ? X[(size_t)row * MLP_IN + f] : 0.f);
  __syncwarp();
  mlp_forward_tile<false>(W, xs[w], MLP_XS, ys[w]);
  mlp_forward_tile<false>(W, xs[w] + 16 * MLP_XS, MLP_XS, ys[w] + 32);
  __syncwarp();
  if (row < n) {
    Y[(size_t)row * 2] = ys[w][l * 2];
    Y[(size_t)row * 2 + 1] = ys[w][l * 2 + 1];
  }
}


}  // namespace

// ---------------------------------------------------------------------------
// harvest of training pairs (one warp per target, uniform traversal)
// ---------------------------------------------------------------------------

namespace {

struct HarvestArgs {
  const NodeF *nodes;
  const FarCell *cells;
  const uint32_t *targets, *idx, *gid, *graphBase, *rootT, *leafPre;
  const double2 *pos;
  const double *mass, *radius;
  float *feat, *tgt, *fmono;
  uint32_t *vert, *cell, *count;
  uint32_t n, cap, maxNodes;
  double kk, overlapC;
  int model;
};

// pair repulsion, reference formulas in FP64 (no coincident pairs here:
// the target is never inside an accepted cell)
__device__ __forceinline__ void pair64(const HarvestArgs &a, double vx, double vy,
                                       double ux, double uy, double mv, double mu,
                                       double rs, double &fx, double &fy) {
  const double dx = ux - vx, dy = uy - vy;
  const double dist = sqrt(dx * dx + dy * dy);
  const double gap = dist - rs;
  const double num = a.model == GVIZ_CUDA_MODEL_FR ? a.kk : mv * mu;
  double mag = gap > 0.0 ? num / gap : num * a.overlapC;
  if (a.model == GVIZ_CUDA_MODEL_FR) mag *= (double)(unsigned long long)mu;
  if (dist > 0.0) {
    fx -= mag * dx / dist;
    fy -= mag * dy / dist;
  }
}

__global__ __launch_bounds__(128) void k_far_harvest(HarvestArgs a) {
  const uint32_t w = (blockIdx.x * 128 + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (w >= a.n) return;
  const uint32_t v = a.targets[w];
  const uint32_t g = a.gid ? a.gid[v] : 0u;
  const uint32_t begin = a.graphBase[g], end = min(begin + a.rootT[g], a.maxNodes);
  const uint32_t myLeaf = a.leafPre[v];
  const double2 p = a.pos[v];
  float vxh, vxl, vyh, vyl;
  ds_split(p.x, vxh, vxl);
  ds_split(p.y, vyh, vyl);
  const double mv = a.mass[v], rv = a.radius[v];
  uint32_t cur = begin;
  while (cur < end) {
    const NodeF n = a.nodes[cur];
    if (n.info >= 0) {  // a single point: evaluated exactly by the walk
      cur++;
      continue;
    }
    const uint32_t next = max((uint32_t)n.next, cur + 1);
    if (n.mass == 0.0f) {
      cur = next;
      continue;
    }
    const float dx = (n.xh - vxh) + (n.xl - vxl);
    const float dy = (n.yh - vyh) + (n.yl - vyl);
    const float d2 = dx * dx + dy * dy;
    const bool containsTarget = cur <= myLeaf && myLeaf < next;
    if (!(n.size < d2) || containsTarget) {
      cur++;
      continue;
    }
    // accepted: exact force of the cell's points (lane-strided, FP64)
    const FarCell c = a.cells[cur];
    double fx = 0.0, fy = 0.0;
    for (uint32_t s = c.s0 + lane; s < c.s1; s += 32) {
      const uint32_t u = a.idx[s];
      const double2 q = a.pos[u];
      pair64(a, p.x, p.y, q.x, q.y, mv, a.mass[u], rv + a.radius[u], fx, fy);
    }
    for (int o = 16; o > 0; o >>= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, o);
      fy += __shfl_xor_sync(0xffffffffu, fy, o);
    }
    if (lane == 0) {
      const double comx = (double)n.xh + (double)n.xl, comy = (double)n.yh + (double)n.yl;
      double mx = 0.0, my = 0.0;
      pair64(a, p.x, p.y, comx, comy, mv, (double)n.mass, rv, mx, my);
      const double fm = sqrt(mx * mx + my * my);
      float f[MLP_IN], e1x, e1y;
      far_features(dx, dy, d2, c, (float)rv, f, e1x, e1y);
      // a pair whose monopole vanishes (FR's pseudo-body mass below one
      // truncates to zero) has no relative correction: not a sample
      const uint32_t slot = fm > 0.0 ? atomicAdd(a.count, 1u) : 0xffffffffu;
      if (slot < a.cap) {
        for (int k = 0; k < MLP_IN; k++) a.feat[(size_t)slot * MLP_IN + k] = f[k];
        const double ex = fx - mx, ey = fy - my;
        a.tgt[(size_t)slot * 2] = (float)((ex * e1x + ey * e1y) / fm);
        a.tgt[(size_t)slot * 2 + 1] = (float)((-ex * e1y + ey * e1x) / fm);
        a.fmono[slot] = (float)fm;
        a.vert[slot] = v;
        a.cell[slot] = cur;
      }
    }
    cur = next;
  }
}

}  // namespace

void mlp_free(gvizCudaForce *h) {
  if (h->d_mlp) cudaFree(h->d_mlp);
  h->d_mlp = nullptr;
}

// far-field side arrays of a handle (allocated on first use)
int far_side_alloc(gvizCudaForce *h) {
  if (h->d_cells) return GVIZ_CUDA_OK;
  const size_t Vs = h->V ? h->V : 1;
  if (cudaMalloc(&h->d_bQ, Vs * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&h->d_nQ, Vs * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&h->d_cells, h->maxNodes * sizeof(FarCell)) != cudaSuccess ||
      cudaMalloc(&h->d_leafPre, Vs * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&h->d_cellCnt, h->maxNodes * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&h->d_groups, Vs * sizeof(uint4)) != cudaSuccess ||
      cudaMalloc(&h->d_groupCount, 2 * sizeof(uint32_t)) != cudaSuccess)
    return GVIZ_CUDA_ERR_ALLOC;
  return GVIZ_CUDA_OK;
}

void far_side_free(gvizCudaForce *h) {
  cudaFree(h->d_bQ);
  cudaFree(h->d_nQ);
  cudaFree(h->d_cells);
  cudaFree(h->d_leafPre);
  cudaFree(h->d_cellCnt);
  cudaFree(h->d_groups);
  cudaFree(h->d_groupCount);
  h->d_bQ = h->d_nQ = nullptr;
  h->d_cells = nullptr;
  h->d_leafPre = nullptr;
  h->d_cellCnt = nullptr;
  h->d_groups = nullptr;
  h->d_groupCount = nullptr;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

int gvizCudaMlpCreate(gvizCudaMlp **out, int device, uint64_t seed) {
  if (!out) return GVIZ_CUDA_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return GVIZ_CUDA_ERR_NO_DEVICE;
  if (device < 0 || device >= ndev) return GVIZ_CUDA_ERR_ARG;
  cudaSetDevice(device);
  gvizCudaMlp *m = new (std::nothrow) gvizCudaMlp();
  if (!m) return GVIZ_CUDA_ERR_ALLOC;
  m->device = device;
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&m->d_w, MLP_PAD * 4) != cudaSuccess ||
      cudaMalloc(&m->d_m, MLP_PAD * 4) != cudaSuccess ||
      cudaMalloc(&m->d_v, MLP_PAD * 4) != cudaSuccess ||
      cudaMalloc(&m->d_dev, sizeof(MlpDev)) != cudaSuccess ||
      cudaMalloc(&m->d_gsum, (MLP_PAD + 1) * 4) != cudaSuccess ||
      cudaMalloc(&m->d_status, 4) != cudaSuccess ||
      cudaMemset(m->d_status, 0, 4) != cudaSuccess) {
    gvizCudaMlpDestroy(m);
    return GVIZ_CUDA_ERR_ALLOC;
  }
  // He-style initialisation from a seeded splitmix stream; zero biases
  std::vector<float> w(MLP_PAD, 0.f);
  uint64_t s = seed * 0x9e3779b97f4a7c15ULL + 1;
  auto uni = [&s]() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return (double)(z >> 11) * 0x1.0p-53 * 2.0 - 1.0;
  };
  for (int j = 0; j < MLP_HID; j++)
    for (int f = 0; f < MLP_IN; f++) w[OFF_W1 + j * MLP_INP + f] = (float)(uni() * sqrt(6.0 / MLP_IN));
  for (int i = 0; i < MLP_HID * MLP_HID; i++) w[OFF_W2 + i] = (float)(uni() * sqrt(6.0 / MLP_HID));
  for (int o = 0; o < MLP_OUT; o++)
    for (int j = 0; j < MLP_HID; j++) w[OFF_W3 + o * MLP_HID + j] = (float)(uni() * 0.1 * sqrt(3.0 / MLP_HID));
  int rc = gvizCudaMlpSetWeights(m, w.data());
  if (rc) {
    gvizCudaMlpDestroy(m);
    return rc;
  }
  *out = m;
  return GVIZ_CUDA_OK;
}

void gvizCudaMlpDestroy(gvizCudaMlp *m) {
  if (!m) return;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->d_w);
  cudaFree(m->d_m);
  cudaFree(m->d_v);
  cudaFree(m->d_dev);
  cudaFree(m->d_grad);
  cudaFree(m->d_gsum);
  cudaFree(m->d_status);
  cudaFree(m->d_epochLoss);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

int gvizCudaMlpParamCount(void) { return MLP_PAD; }

int gvizCudaMlpSetTrainingKernels(gvizCudaMlp *m, int tcgen05) {
  if (!m || (tcgen05 != 0 && tcgen05 != 1)) return GVIZ_CUDA_ERR_ARG;
  m->tc = tcgen05 != 0;
  return GVIZ_CUDA_OK;
}

int gvizCudaMlpSetWeights(gvizCudaMlp *m, const float *w) {
  if (!m || !w) return GVIZ_CUDA_ERR_ARG;
  cudaSetDevice(m->device);
  if (cudaMemcpy(m->d_w, w, MLP_PAD * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(m->d_m, 0, MLP_PAD * 4) != cudaSuccess ||
      cudaMemset(m->d_v, 0, MLP_PAD * 4) != cudaSuccess)
    return GVIZ_CUDA_ERR_CUDA;
  m->step = 0;
  k_mlp_to_dev<<<(MLP_PAD + 255) / 256, 256, 0, m->stream>>>(m->d_w, m->d_dev);
  return cudaStreamSynchronize(m->stream) == cudaSuccess ? GVIZ_CUDA_OK : GVIZ_CUDA_ERR_CUDA;
}

int gvizCudaMlpGetWeights(gvizCudaMlp *m, float *w) {
  if (!m || !w) return GVIZ_CUDA_ERR_ARG;
  cudaSetDevice(m->device);
  cudaStreamSynchronize(m->stream);
  return cudaMemcpy(w, m->d_w, MLP_PAD * 4, cudaMemcpyDeviceToHost) == cudaSuccess
             ? GVIZ_CUDA_OK : GVIZ_CUDA_ERR_CUDA;
}

static int mlp_grad_launch(gvizCudaMlp *m, const float *dX, const float *dT,
                           const float *dW, const uint32_t *dOrder, uint32_t n,
                           float scale) {
  const uint32_t tiles = m->tc ? (n + kTcThreads - 1) / kTcThreads : (n + 31) / 32;
  const uint32_t per = m->tc ? kTcTilesPerBlock : kTilesPerBlock;
  const uint32_t blocks = (tiles + per - 1) / per;
  if (blocks > m->gradBlocks) {
    cudaFree(m->d_grad);
    m->d_grad = nullptr;
    if (cudaMalloc(&m->d_grad, (size_t)blocks * (MLP_PAD + 1) * 4) != cudaSuccess)
      return GVIZ_CUDA_ERR_ALLOC;
    m->gradBlocks = blocks;
  }
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(TrainSmem));
    cudaFuncSetAttribute(k_mlp_grad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(TcSmem));
    attr = true;
  }
  if (m->tc)
    k_mlp_grad_tc<<<blocks, kTcThreads, sizeof(TcSmem), m->stream>>>(
        m->d_w, dX, dT, dW, dOrder, n, scale, m->d_grad, m->d_status);
  else
    k_mlp_grad<<<blocks, 32, sizeof(TrainSmem), m->stream>>>(m->d_w, dX, dT, dW, dOrder, n,
                                                             scale, m->d_grad);
  k_mlp_reduce<<<(MLP_PAD + 1 + 255) / 256, 256, 0, m->stream>>>(m->d_grad, blocks, m->d_gsum);
  return GVIZ_CUDA_OK;
}

// After a synchronisation: GVIZ_CUDA_ERR_CUDA when a tcgen05 kernel gave up
// waiting for its tensor-core work (status cleared for the next call).
static int mlp_status(gvizCudaMlp *m) {
  uint32_t st = 0;
  if (cudaMemcpy(&st, m->d_status, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return GVIZ_CUDA_ERR_CUDA;
  if (st) {
    cudaMemset(m->d_status, 0, 4);
    return GVIZ_CUDA_ERR_CUDA;
  }
  return GVIZ_CUDA_OK;
}

// Gradient of the weighted mean squared error over n samples (host arrays:
// X n*10, T n*2, W n or NULL for unit weights). grad: MLP_PAD floats in the
// master layout; loss: the weighted mean.
int gvizCudaMlpGradient(gvizCudaMlp *m, const float *X, const float *T,
                        const float *W, size_t n, float *grad, float *loss) {
  if (!m || !X || !T || n == 0) return GVIZ_CUDA_ERR_ARG;
  cudaSetDevice(m->device);
  float *dX, *dT, *dW = nullptr;
  double wsum = 0.0;
  for (size_t i = 0; i < n; i++) wsum += W ? W[i] : 1.0;
  if (cudaMalloc(&dX, n * MLP_IN * 4) != cudaSuccess || cudaMalloc(&dT, n * 8) != cudaSuccess)
    return GVIZ_CUDA_ERR_ALLOC;
  cudaMemcpy(dX, X, n * MLP_IN * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dT, T, n * 8, cudaMemcpyHostToDevice);
  if (W) {
    cudaMalloc(&dW, n * 4);
    cudaMemcpy(dW, W, n * 4, cudaMemcpyHostToDevice);
  }
  int rc = mlp_grad_launch(m, dX, dT, dW, nullptr, (uint32_t)n, (float)(1.0 / wsum));
  std::vector<float> gs(MLP_PAD + 1);
  if (!rc && cudaMemcpyAsync(gs.data(), m->d_gsum, (MLP_PAD + 1) * 4, cudaMemcpyDeviceToHost,
                             m->stream) == cudaSuccess &&
      cudaStreamSynchronize(m->stream) == cudaSuccess) {
    rc = mlp_status(m);
    if (!rc && grad) memcpy(grad, gs.data(), MLP_PAD * 4);
    if (!rc && loss) *loss = gs[MLP_PAD];
  } else if (!rc) {
    rc = GVIZ_CUDA_ERR_CUDA;
  }
  cudaFree(dX);
  cudaFree(dT);
  cudaFree(dW);
  return rc;
}

// Adam training on n samples (host arrays as in gvizCudaMlpGradient):
// `epochs` passes in mini-batches of `batch`, samples shuffled per epoch
// with a seeded permutation. lossOut[epochs] (may be NULL) receives each
// epoch's mean training loss.
int gvizCudaMlpTrain(gvizCudaMlp *m, const float *X, const float *T,
                     const float *W, size_t n, uint32_t epochs, uint32_t batch,
                     float lr, uint64_t seed, float *lossOut) {
  if (!m || !X || !T || n == 0 || batch == 0) return GVIZ_CUDA_ERR_ARG;
  cudaSetDevice(m->device);
  float *dX = nullptr, *dT = nullptr, *dW = nullptr;
  uint32_t *dOrder = nullptr;
  int rc = GVIZ_CUDA_OK;
  if (cudaMalloc(&dX, n * MLP_IN * 4) != cudaSuccess || cudaMalloc(&dT, n * 8) != cudaSuccess ||
      cudaMalloc(&dOrder, n * 4) != cudaSuccess || (W && cudaMalloc(&dW, n * 4) != cudaSuccess))
    rc = GVIZ_CUDA_ERR_ALLOC;
  std::vector<float> wn;
  if (!rc) {
    cudaMemcpy(dX, X, n * MLP_IN * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dT, T, n * 8, cudaMemcpyHostToDevice);
    if (W) cudaMemcpy(dW, W, n * 4, cudaMemcpyHostToDevice);
  }
  std::vector<uint32_t> order(n);
  for (size_t i = 0; i < n; i++) order[i] = (uint32_t)i;
  uint64_t s = seed ^ 0xD1B54A32D192ED03ULL;
  auto rnd = [&s]() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  };
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  // the epochs' losses are summed on the device (no synchronisation per
  // mini-batch) and read once at the end
  if (!rc && lossOut && epochs > m->epochCap) {
    cudaFree(m->d_epochLoss);
    m->d_epochLoss = nullptr;
    m->epochCap = 0;
    if (cudaMalloc(&m->d_epochLoss, epochs * sizeof(float)) != cudaSuccess)
      rc = GVIZ_CUDA_ERR_ALLOC;
    else
      m->epochCap = epochs;
  }
  if (!rc && lossOut) cudaMemsetAsync(m->d_epochLoss, 0, epochs * sizeof(float), m->stream);
  // one pinned staging buffer for the per-epoch order upload
  uint32_t *hOrder = nullptr;
  if (!rc && cudaMallocHost(&hOrder, n * 4) != cudaSuccess) rc = GVIZ_CUDA_ERR_ALLOC;
  for (uint32_t ep = 0; ep < epochs && !rc; ep++) {
    for (size_t i = n - 1; i > 0; i--) std::swap(order[i], order[rnd() % (i + 1)]);
    cudaStreamSynchronize(m->stream);  // the previous epoch's upload is done
    memcpy(hOrder, order.data(), n * 4);
    cudaMemcpyAsync(dOrder, hOrder, n * 4, cudaMemcpyHostToDevice, m->stream);
    for (size_t b0 = 0; b0 < n && !rc; b0 += batch) {
      const uint32_t nb = (uint32_t)std::min<size_t>(batch, n - b0);
      double wsum = 0.0;
      for (uint32_t i = 0; i < nb; i++) wsum += W ? W[order[b0 + i]] : 1.0;
      rc = mlp_grad_launch(m, dX, dT, dW, dOrder + b0, nb, (float)(1.0 / wsum));
      if (rc) break;
      m->step++;
      const float c1 = 1.f - powf(b1, (float)m->step), c2 = 1.f - powf(b2, (float)m->step);
      k_mlp_adam<<<(MLP_PAD + 255) / 256, 256, 0, m->stream>>>(
          m->d_w, m->d_m, m->d_v, m->d_gsum, lr, b1, b2, eps, c1, c2,
          lossOut ? m->d_epochLoss + ep : nullptr, (float)nb);
    }
  }
  k_mlp_to_dev<<<(MLP_PAD + 255) / 256, 256, 0, m->stream>>>(m->d_w, m->d_dev);
  if (cudaStreamSynchronize(m->stream) != cudaSuccess && !rc) rc = GVIZ_CUDA_ERR_CUDA;
  if (!rc) rc = mlp_status(m);
  if (!rc && lossOut) {
    std::vector<float> el(epochs);
    if (cudaMemcpy(el.data(), m->d_epochLoss, epochs * sizeof(float), cudaMemcpyDeviceToHost) !=
        cudaSuccess)
      rc = GVIZ_CUDA_ERR_CUDA;
    for (uint32_t ep = 0; ep < epochs && !rc; ep++) lossOut[ep] = (float)(el[ep] / (double)n);
  }
  cudaFreeHost(hOrder);
  cudaFree(dX);
  cudaFree(dT);
  cudaFree(dW);
  cudaFree(dOrder);
  return rc;
}

// Batch inference with the BF16 tensor-core forward pass: Y (n*2) from X (n*10).
int gvizCudaMlpInfer(gvizCudaMlp *m, const float *X, size_t n, float *Y) {
  if (!m || !X || !Y) return GVIZ_CUDA_ERR_ARG;
  if (n == 0) return GVIZ_CUDA_OK;
  cudaSetDevice(m->device);
  float *dX, *dY;
  if (cudaMalloc(&dX, n * MLP_IN * 4) != cudaSuccess || cudaMalloc(&dY, n * 8) != cudaSuccess)
    return GVIZ_CUDA_ERR_ALLOC;
  cudaMemcpy(dX, X, n * MLP_IN * 4, cudaMemcpyHostToDevice);
  const uint32_t blocks = (uint32_t)((n + 127) / 128);
  k_mlp_infer<<<blocks, 128, 0, m->stream>>>(m->d_dev, dX, (uint32_t)n, dY);
  int rc = cudaStreamSynchronize(m->stream) == cudaSuccess ? GVIZ_CUDA_OK : GVIZ_CUDA_ERR_CUDA;
  if (!rc) cudaMemcpy(Y, dY, n * 8, cudaMemcpyDeviceToHost);
  cudaFree(dX);
  cudaFree(dY);
  return rc;
}

// Attaches a trained model to a layout (copies its BF16 weights).
int gvizCudaForceSetFarFieldModel(gvizCudaForce *h, gvizCudaMlp *m) {
  if (!h) return GVIZ_CUDA_ERR_ARG;
  cudaSetDevice(h->device);
  if (!m) {
    mlp_free(h);
    h->params.farField = 0;  // nothing to apply any more
    h->farSide = false;
    h->graphDirty = true;
    return GVIZ_CUDA_OK;
  }
  if (!h->d_mlp && cudaMalloc(&h->d_mlp, sizeof(MlpDev)) != cudaSuccess)
    return GVIZ_CUDA_ERR_ALLOC;
  cudaStreamSynchronize(m->stream);
  if (cudaMemcpy(h->d_mlp, m->d_dev, sizeof(MlpDev), cudaMemcpyDeviceToDevice) != cudaSuccess)
    return GVIZ_CUDA_ERR_CUDA;
  int rc = far_side_alloc(h);
  h->graphDirty = true;
  return rc;
}

// The target groups of the learned cell-group walk on the current positions
// (built as a step builds them): per vertex the index of its group.
int gvizCudaForceFarGroups(gvizCudaForce *h, uint32_t *groupOf, uint64_t *groupCount) {
  if (!h || (h->V && !groupOf) || !groupCount) return GVIZ_CUDA_ERR_ARG;
  cudaSetDevice(h->device);
  *groupCount = 0;
  if (!h->V) return GVIZ_CUDA_OK;
  int rc = far_side_alloc(h);
  if (rc) return rc;
  const gvizCudaForceParams saved = h->params;
  h->params.precision = GVIZ_CUDA_FP32;
  h->params.farCellGroups = 1;
  const bool savedSide = h->farSide;
  h->farSide = true;
  cudaMemsetAsync(h->d_status, 0, 4, h->stream);
  enqueue_tree_build(h);
  h->farSide = savedSide;
  h->params = saved;
  uint32_t *dOut = nullptr, count = 0, status = 0;
  if (cudaMalloc(&dOut, h->V * 4) != cudaSuccess) return GVIZ_CUDA_ERR_ALLOC;
  cudaMemsetAsync(dOut, 0xff, h->V * 4, h->stream);
  enqueue_group_export(h, dOut);
  cudaMemcpyAsync(groupOf, dOut, h->V * 4, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(&count, h->d_groupCount, 4, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(&status, h->d_status, 4, cudaMemcpyDeviceToHost, h->stream);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) rc = GVIZ_CUDA_ERR_CUDA;
  cudaFree(dOut);
  if (!rc && status) rc = GVIZ_CUDA_ERR_LIMIT;
  *groupCount = count;
  return rc;
}

// Training pairs for the learned correction at opening threshold `theta`
// on the current positions: for each listed target vertex, every accepted
// cell gives features[10], the relative correction target[2] in the pair
// frame, the monopole magnitude and the target vertex. Returns the number of
// pairs found (may exceed cap; only cap are written).
int64_t gvizCudaForceHarvestFarField(gvizCudaForce *h, const uint32_t *targets,
                                     size_t nTargets, double theta, float *features,
                                     float *target, float *fmono, uint32_t *vertex,
                                     size_t cap) {
  if (!h || (nTargets && !targets)) return GVIZ_CUDA_ERR_ARG;
  cudaSetDevice(h->device);
  int rc = far_side_alloc(h);
  if (rc) return rc;
  const gvizCudaForceParams saved = h->params;
  h->params.theta = theta;
  h->params.precision = GVIZ_CUDA_FP32;
  const bool savedSide = h->farSide;
  h->farSide = true;
  cudaMemsetAsync(h->d_status, 0, 4, h->stream);
  enqueue_tree_build(h);
  h->farSide = savedSide;
  h->params = saved;
  uint32_t *dT = nullptr, *dCount = nullptr, *dV = nullptr, *dC = nullptr;
  float *dF = nullptr, *dG = nullptr, *dM = nullptr;
  const size_t c = cap ? cap : 1;
  if (cudaMalloc(&dT, (nTargets ? nTargets : 1) * 4) != cudaSuccess ||
      cudaMalloc(&dCount, 4) != cudaSuccess || cudaMalloc(&dF, c * MLP_IN * 4) != cudaSuccess ||
      cudaMalloc(&dG, c * 8) != cudaSuccess || cudaMalloc(&dM, c * 4) != cudaSuccess ||
      cudaMalloc(&dV, c * 4) != cudaSuccess || cudaMalloc(&dC, c * 4) != cudaSuccess) {
    rc = GVIZ_CUDA_ERR_ALLOC;
  }
  uint32_t count = 0;
  if (!rc) {
    cudaMemcpyAsync(dT, targets, nTargets * 4, cudaMemcpyHostToDevice, h->stream);
    cudaMemsetAsync(dCount, 0, 4, h->stream);
    HarvestArgs a;
    a.nodes = reinterpret_cast<const NodeF *>(h->d_nodes);
    a.cells = h->d_cells;
    a.targets = dT;
    a.idx = h->d_idx;
    a.gid = h->d_gid;
    a.graphBase = h->d_graphBase;
    a.rootT = h->d_rootT;
    a.leafPre = h->d_leafPre;
    a.pos = h->d_pos;
    a.mass = h->d_mass;
    a.radius = h->d_radius;
    a.feat = dF;
    a.tgt = dG;
    a.fmono = dM;
    a.vert = dV;
    a.cell = dC;
    a.count = dCount;
    a.n = (uint32_t)nTargets;
    a.cap = (uint32_t)cap;
    a.maxNodes = (uint32_t)h->maxNodes;
    a.kk = h->params.edgeLength * h->params.edgeLength;
    a.overlapC = h->params.overlapConstant;
    a.model = h->model;
    if (nTargets)
      k_far_harvest<<<(uint32_t)((nTargets * 32 + 127) / 128), 128, 0, h->stream>>>(a);
    cudaMemcpyAsync(&count, dCount, 4, cudaMemcpyDeviceToHost, h->stream);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) rc = GVIZ_CUDA_ERR_CUDA;
  }
  if (!rc && count > 0 && count <= cap) {
    // the kernel appends in scheduling order; return the pairs in one
    // canonical order (target vertex, then cell) so that results built on
    // them (training) do not depend on it
    const size_t n = count;
    std::vector<float> F(n * MLP_IN), G(n * 2), M(n);
    std::vector<uint32_t> Vv(n), Cc(n), perm(n);
    bool ok = cudaMemcpy(F.data(), dF, n * MLP_IN * 4, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(G.data(), dG, n * 8, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(M.data(), dM, n * 4, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(Vv.data(), dV, n * 4, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(Cc.data(), dC, n * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (!ok) rc = GVIZ_CUDA_ERR_CUDA;
    for (size_t i = 0; i < n; i++) perm[i] = (uint32_t)i;
    std::sort(perm.begin(), perm.end(), [&](uint32_t x, uint32_t y) {
      return Vv[x] != Vv[y] ? Vv[x] < Vv[y] : Cc[x] < Cc[y];
    });
    for (size_t o = 0; !rc && o < n; o++) {
      const uint32_t i = perm[o];
      if (features) memcpy(features + o * MLP_IN, &F[i * MLP_IN], MLP_IN * 4);
      if (target) memcpy(target + 2 * o, &G[2 * i], 8);
      if (fmono) fmono[o] = M[i];
      if (vertex) vertex[o] = Vv[i];
    }
  }
  cudaFree(dC);
  cudaFree(dT);
  cudaFree(dCount);
  cudaFree(dF);
  cudaFree(dG);
  cudaFree(dM);
  cudaFree(dV);
  return rc ? (int64_t)rc : (int64_t)count;
}

}  // extern "C"
