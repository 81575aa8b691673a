// mlp.cuh -- the learned far-field correction: features of a (target, cell)
// pair, the 10 -> 64 -> 64 -> 2 MLP on BF16 tensor cores (FP32 accumulate),
// shared by training (mlp.cu) and the fused walk (forces.cu).
//
// The Barnes-Hut pseudo-body force of a cell (mass M, centre of mass c) on a
// target v is the monopole term; for the 1/r pair kernels of FR and LinLog
// the leading correction is the cell's quadrupole over |c - v|^2, then
// higher multipoles. The MLP predicts the relative correction in the local
// frame of the pair (e1 = direction of the monopole force, e2 = e1 rotated
// by +90 degrees) in units of its leading order s^2 = (h/d)^2:
//     F = F_mono + |F_mono| s^2 (m1 e1 + m2 e2),   m = MLP(features)
// from rotation-invariant features (the quadrupole is rotated into the same
// frame), so one small network serves every direction and every distance.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "internal.cuh"

#define MLP_IN 10
#define MLP_INP 16  // input padded to one k-tile
#define MLP_HID 64
#define MLP_OUT 2
#define MLP_OUTP 8  // output padded to one n-tile
// parameter count: 10*64 + 64 + 64*64 + 64 + 64*2 + 2 = 4994
#define MLP_PARAMS (MLP_IN * MLP_HID + MLP_HID + MLP_HID * MLP_HID + MLP_HID + MLP_HID * MLP_OUT + MLP_OUT)

// Device weights for the tensor-core kernels: transposed ([out][in], in
// contiguous) BF16 matrices padded to MMA tiles, FP32 biases.
struct __align__(16) MlpDev {
  __nv_bfloat16 w1t[MLP_HID * MLP_INP];   // [64][16]
  __nv_bfloat16 w2t[MLP_HID * MLP_HID];   // [64][64]
  __nv_bfloat16 w3t[MLP_OUTP * MLP_HID];  // [8][64]
  float b1[MLP_HID];
  float b2[MLP_HID];
  float b3[MLP_OUTP];
};

// Shared-memory row strides for ldmatrix operands: 48-byte rows (16 BF16
// used) and 144-byte rows (64 used) put the eight 16-byte row segments of
// one 8x8 matrix in eight different bank groups (a 32- or 128-byte stride
// would serialise them 2- or 8-way).
#define MLP_XS 24
#define MLP_HS 72

// The inference weights as staged in shared memory by mlp_stage.
struct __align__(16) MlpSmem {
  __nv_bfloat16 w1t[MLP_HID * MLP_XS];
  __nv_bfloat16 w2t[MLP_HID * MLP_HS];
  __nv_bfloat16 w3t[MLP_OUTP * MLP_HS];
  float b1[MLP_HID];
  float b2[MLP_HID];
  float b3[MLP_OUTP];
};

// Whole-block copy of the device weights into the padded layout; the caller
// synchronises the block afterwards.
__device__ __forceinline__ void mlp_stage(MlpSmem &S, const MlpDev *__restrict__ g) {
  const uint32_t *w1 = reinterpret_cast<const uint32_t *>(g->w1t);
  const uint32_t *w2 = reinterpret_cast<const uint32_t *>(g->w2t);
  const uint32_t *w3 = reinterpret_cast<const uint32_t *>(g->w3t);
  uint32_t *s1 = reinterpret_cast<uint32_t *>(S.w1t);
  uint32_t *s2 = reinterpret_cast<uint32_t *>(S.w2t);
  uint32_t *s3 = reinterpret_cast<uint32_t *>(S.w3t);
  for (int i = threadIdx.x; i < MLP_HID * MLP_INP / 2; i += blockDim.x)
    s1[(i / (MLP_INP / 2)) * (MLP_XS / 2) + i % (MLP_INP / 2)] = __ldg(w1 + i);
  for (int i = threadIdx.x; i < MLP_HID * MLP_HID / 2; i += blockDim.x)
    s2[(i / (MLP_HID / 2)) * (MLP_HS / 2) + i % (MLP_HID / 2)] = __ldg(w2 + i);
  for (int i = threadIdx.x; i < MLP_OUTP * MLP_HID / 2; i += blockDim.x)
    s3[(i / (MLP_HID / 2)) * (MLP_HS / 2) + i % (MLP_HID / 2)] = __ldg(w3 + i);
  for (int i = threadIdx.x; i < MLP_HID; i += blockDim.x) {
    S.b1[i] = __ldg(g->b1 + i);
    S.b2[i] = __ldg(g->b2 + i);
  }
  for (int i = threadIdx.x; i < MLP_OUTP; i += blockDim.x) S.b3[i] = __ldg(g->b3 + i);
}

// ---------------------------------------------------------------------------
// features
// ---------------------------------------------------------------------------

// (dx, dy) = c - v, d2 = |c - v|^2 (FP32), FarCell of the accepted cell,
// target radius rv (0 without overlap). Writes the 10 features and the
// frame (e1 = -(c-v)/|c-v|).
__device__ __forceinline__ void far_features(float dx, float dy, float d2,
                                             const FarCell &c, float rv, float *f,
                                             float &e1x, float &e1y) {
  const float inv = rsqrtf(d2);
  const float inv2 = inv * inv;
  const float wx = dx * inv, wy = dy * inv;  // unit vector v -> c
  e1x = -wx;
  e1y = -wy;
  // quadrupole (Qxx - Qyy) + 2i Qxy rotated by conj(w)^2 into the pair frame
  const float ca = wx * wx - wy * wy, cb = -2.0f * wx * wy;
  const float s = c.h * inv;  // h / d
  f[0] = s;
  f[1] = (c.qa * ca - c.qb * cb) * inv2;
  f[2] = (c.qa * cb + c.qb * ca) * inv2;
  f[3] = c.tr * inv2;
  f[4] = rv * inv;
  f[5] = c.ox * wx + c.oy * wy;
  f[6] = c.oy * wx - c.ox * wy;
  f[7] = __log2f((float)max(c.s1 - c.s0, 1u)) * (1.0f / 16.0f);
  f[8] = s * s;
  f[9] = s * s * s;
}

// ---------------------------------------------------------------------------
// tensor-core fragments (mma.sync m16n8k16, BF16 in, FP32 accumulate)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ void mma16816(float *c, const uint32_t *a,
                                         const uint32_t *b) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void ldsm_x4(uint32_t *r, const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t *r, const void *p) {
  asm volatile(
      "ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
      : "r"(smem_u32(p)));
}

__device__ __forceinline__ void ldsm_x2(uint32_t *r, const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n"
               : "=r"(r[0]), "=r"(r[1])
               : "r"(smem_u32(p)));
}

__device__ __forceinline__ void ldsm_x2_t(uint32_t *r, const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
               : "=r"(r[0]), "=r"(r[1])
               : "r"(smem_u32(p)));
}

// A fragment (16x16) at (row0, col0) of a row-major BF16 matrix with `ld`
// elements per row.
__device__ __forceinline__ void load_a(uint32_t *a, const __nv_bfloat16 *m,
                                       int ld, int row0, int col0) {
  const int l = threadIdx.x & 31;
  const int r = l & 7, j = l >> 3;
  const __nv_bfloat16 *p = m + (row0 + r + ((j & 1) << 3)) * ld + col0 + ((j >> 1) << 3);
  ldsm_x4(a, p);
}

// A fragment of the TRANSPOSE of a row-major matrix S ([k][m] in memory):
// A[m][k] = S[k][m], tile at (m0, k0).
__device__ __forceinline__ void load_a_t(uint32_t *a, const __nv_bfloat16 *s,
                                         int ld, int m0, int k0) {
  const int l = threadIdx.x & 31;
  const int r = l & 7, j = l >> 3;
  // matrices: (m0..+7, k0..+7), (m0+8.., k0..), (m0.., k0+8..), (m0+8.., k0+8..)
  const __nv_bfloat16 *p = s + (k0 + r + ((j >> 1) << 3)) * ld + m0 + ((j & 1) << 3);
  ldsm_x4_t(a, p);
}

// B fragment (16x8, k x n) from a matrix stored [n][k] (k contiguous):
// the transposed-weight layout. Tile at (k0, n0).
__device__ __forceinline__ void load_b_nk(uint32_t *b, const __nv_bfloat16 *m,
                                          int ld, int k0, int n0) {
  const int l = threadIdx.x & 15;
  const int r = l & 7, j = l >> 3;
  const __nv_bfloat16 *p = m + (n0 + r) * ld + k0 + (j << 3);
  ldsm_x2(b, p);
}

// B fragment (16x8, k x n) from a row-major matrix stored [k][n].
__device__ __forceinline__ void load_b_kn(uint32_t *b, const __nv_bfloat16 *m,
                                          int ld, int k0, int n0) {
  const int l = threadIdx.x & 15;
  const int r = l & 7, j = l >> 3;
  const __nv_bfloat16 *p = m + (k0 + r + (j << 3)) * ld + n0;
  ldsm_x2_t(b, p);
}

// B fragments of two adjacent n-tiles (16x16, k x n) from a matrix stored
// [n][k] (k contiguous), one ldmatrix.x4: b[0..1] n-tile n0, b[2..3] n0 + 8.
__device__ __forceinline__ void load_b2_nk(uint32_t *b, const __nv_bfloat16 *m,
                                           int ld, int k0, int n0) {
  const int l = threadIdx.x & 31;
  const int r = l & 7, j = l >> 3;
  const __nv_bfloat16 *p = m + (n0 + r + ((j >> 1) << 3)) * ld + k0 + ((j & 1) << 3);
  ldsm_x4(b, p);
}

// Forward pass of one 16-row tile: X (16 rows of 16 BF16 features in shared
// memory, row stride ldx) -> out[16][2] FP32 in shared memory. W holds the
// weights staged by mlp_stage. Hidden layers stay in registers: the
// accumulator layout of two adjacent n-tiles is the A layout of one k-tile.
// With SCALE_S2 the outputs are multiplied by the row's feature 8, s^2: the
// network predicts the relative correction in units of (h/d)^2, its leading
// order, so the correction vanishes with the cell's angular size.
template <bool SCALE_S2>
__device__ __forceinline__ void mlp_forward_tile(const MlpSmem &W,
                                                 const __nv_bfloat16 *X, int ldx,
                                                 float *out) {
  const int l = threadIdx.x & 31;
  const int g = l >> 2, t = l & 3;
  uint32_t a[4];
  load_a(a, X, ldx, 0, 0);
  // layer 1: 8 n-tiles of 8 hidden units
  uint32_t h1[4][4];  // A fragments of layer 2 (4 k-tiles)
#pragma unroll
  for (int kt = 0; kt < 4; kt++) {
    float c0[4] = {0.f, 0.f, 0.f, 0.f}, c1[4] = {0.f, 0.f, 0.f, 0.f};
    uint32_t b[4];
    load_b2_nk(b, W.w1t, MLP_XS, 0, 16 * kt);
    mma16816(c0, a, b);
    mma16816(c1, a, b + 2);
    const int n0 = 16 * kt + 2 * t, n1 = n0 + 8;
    const float b00 = W.b1[n0], b01 = W.b1[n0 + 1], b10 = W.b1[n1], b11 = W.b1[n1 + 1];
    h1[kt][0] = pack_bf16(fmaxf(c0[0] + b00, 0.f), fmaxf(c0[1] + b01, 0.f));
    h1[kt][1] = pack_bf16(fmaxf(c0[2] + b00, 0.f), fmaxf(c0[3] + b01, 0.f));
    h1[kt][2] = pack_bf16(fmaxf(c1[0] + b10, 0.f), fmaxf(c1[1] + b11, 0.f));
    h1[kt][3] = pack_bf16(fmaxf(c1[2] + b10, 0.f), fmaxf(c1[3] + b11, 0.f));
  }
  // layers 2 and 3 interleaved: each pair of layer-2 n-tiles becomes one
  // k-tile of layer 3 right away
  float y[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int kt3 = 0; kt3 < 4; kt3++) {
    float c0[4] = {0.f, 0.f, 0.f, 0.f}, c1[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kt = 0; kt < 4; kt++) {
      uint32_t b[4];
      load_b2_nk(b, W.w2t, MLP_HS, 16 * kt, 16 * kt3);
      mma16816(c0, h1[kt], b);
      mma16816(c1, h1[kt], b + 2);
    }
    const int n0 = 16 * kt3 + 2 * t, n1 = n0 + 8;
    const float b00 = W.b2[n0], b01 = W.b2[n0 + 1], b10 = W.b2[n1], b11 = W.b2[n1 + 1];
    uint32_t h2[4];
    h2[0] = pack_bf16(fmaxf(c0[0] + b00, 0.f), fmaxf(c0[1] + b01, 0.f));
    h2[1] = pack_bf16(fmaxf(c0[2] + b00, 0.f), fmaxf(c0[3] + b01, 0.f));
    h2[2] = pack_bf16(fmaxf(c1[0] + b10, 0.f), fmaxf(c1[1] + b11, 0.f));
    h2[3] = pack_bf16(fmaxf(c1[2] + b10, 0.f), fmaxf(c1[3] + b11, 0.f));
    uint32_t b[2];
    load_b_nk(b, W.w3t, MLP_HS, 16 * kt3, 0);
    mma16816(y, h2, b);
  }
  // outputs 0 and 1 sit in threads with t == 0: rows g and g + 8
  if (t == 0) {
    const float s0 = SCALE_S2 ? __bfloat162float(X[g * ldx + 8]) : 1.f;
    const float s1 = SCALE_S2 ? __bfloat162float(X[(g + 8) * ldx + 8]) : 1.f;
    out[g * 2 + 0] = (y[0] + W.b3[0]) * s0;
    out[g * 2 + 1] = (y[1] + W.b3[1]) * s0;
    out[(g + 8) * 2 + 0] = (y[2] + W.b3[0]) * s1;
    out[(g + 8) * 2 + 1] = (y[3] + W.b3[1]) * s1;
  }
}
