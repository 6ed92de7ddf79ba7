// Per-particle MLP of the learned warm start: 12 -> 64 -> 64 -> 1, GELU
// (erf form), BF16 weights and activations on the tensor cores, FP32
// accumulation (mma.sync.m16n8k16.row.col.f32.bf16.bf16.f32).
//
// A warp evaluates a tile of 16 particles.  Fragment layouts (PTX ISA,
// m16n8k16, g = lane/4, t = lane%4):
//   A 16x16 row-major, 4 x b32:  a0 (g, 2t..2t+1)   a1 (g+8, 2t..2t+1)
//                                a2 (g, 2t+8..+9)   a3 (g+8, 2t+8..+9)
//   B 16x8 column-major, 2 x b32: b0 (2t..2t+1, g)  b1 (2t+8..+9, g)
//   C/D 16x8, 4 x f32:           (g, 2t) (g, 2t+1) (g+8, 2t) (g+8, 2t+1)
// The D fragments of two neighbouring 8-column tiles are exactly the A
// fragment of the next layer's 16-wide k step, so activations stay in
// registers between layers.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace pbf {

constexpr int kMlpIn = 12;       // features
constexpr int kMlpInPad = 16;    // k of the first layer
constexpr int kMlpH = 64;        // hidden width
// fp32 master parameters, canonical order:
//   W1[64][12] (row = output unit), b1[64], W2[64][64] (row = output unit),
//   b2[64], w3[64], b3
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpH * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpH;
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH;
constexpr int kOffB3 = kOffW3 + kMlpH;
constexpr int kMlpParams = kOffB3 + 1;  // 5057

// Device copy of the network used by the kernels.
struct MlpDev {
  const __nv_bfloat16* w1;   // [64][16]  W1 padded (k = 12..15 zero): B operand of layer 1
  const __nv_bfloat16* w2;   // [64][64]  W2 as stored (n-major): B operand of layer 2
  const __nv_bfloat16* w2t;  // [64][64]  W2 transposed (k-major): B operand of dH1 = dZ2 W2
  const float* b1;
  const float* b2;
  const float* w3;
  const float* b3;
  const float* feat_mean;    // [12] feature normalisation: (f - mean) * inv_std
  const float* feat_inv_std; // [12]
  float label_scale;         // lambda = y * label_scale
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float d[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// GELU(x) = x/2 (1 + erf(x/sqrt 2)) and its derivative.
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.3989422804014327f * __expf(-0.5f * x * x);
  return cdf + x * pdf;
}

// GELU of two values at once for the tensor-core network's epilogues:
// x/2 (1 + erf(u)), u = x/sqrt 2 clamped to [-3, 3], erf(u) = u q(u^2) with q a
// degree-8 polynomial fitted to erf on [0, 3] (iteratively reweighted least
// squares on Chebyshev nodes, this project's own fit).  In float32 its error is
// below 2.7e-5 in erf (the clamp's 1 - erf(3) = 2.2e-5 included) and 6e-5 in
// GELU, far under the bf16 rounding (2^-9) of the activations it feeds.  The
// packed f32x2 operations evaluate two GELUs per instruction.
__device__ __forceinline__ float2 gelu2(float2 x) {
  constexpr float kErfQ[9] = {1.1282683610916138f,    -0.3753148019313812f,   0.11107926070690155f,
                              -0.025102820247411728f, 0.0042354147881269455f, -0.0005110346246510744f,
                              4.106029155082069e-05f, -1.944809810083825e-06f, 4.0741806373034706e-08f};
  float2 u = __fmul2_rn(x, make_float2(0.70710678118654752f, 0.70710678118654752f));
  u.x = fminf(fmaxf(u.x, -3.0f), 3.0f);
  u.y = fminf(fmaxf(u.y, -3.0f), 3.0f);
  const float2 u2 = __fmul2_rn(u, u);
  float2 q = make_float2(kErfQ[8], kErfQ[8]);
#pragma unroll
  for (int k = 7; k >= 0; --k) q = __ffma2_rn(q, u2, make_float2(kErfQ[k], kErfQ[k]));
  const float2 e = __fmul2_rn(q, u);
  const float2 hx = __fmul2_rn(x, make_float2(0.5f, 0.5f));
  return __ffma2_rn(hx, e, hx);
}

// B fragment of an [n][k]-stored (n-major, k contiguous) bf16 matrix with row
// stride ld, for the 8-column tile n0 and the 16-deep k step k0.
__device__ __forceinline__ void load_b(uint32_t b[2], const __nv_bfloat16* w, int ld, int n0, int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const __nv_bfloat16* p = w + (size_t)(n0 + g) * ld + k0 + 2 * t;
  b[0] = *reinterpret_cast<const uint32_t*>(p);
  b[1] = *reinterpret_cast<const uint32_t*>(p + 8);
}

// Forward pass of one 16-row tile.  a_in: A fragment of the normalised,
// zero-padded features.  Returns y for rows g and g+8 (every lane of a quad
// holds the same two values).  When z1/z2 are given, the pre-activations are
// kept (D layout, 8 tiles x 4) for the backward pass.
__device__ __forceinline__ void mlp_forward16(const MlpDev& M, const uint32_t a_in[4], int lane, float& y_lo,
                                              float& y_hi, float (*z1)[4] = nullptr, float (*z2)[4] = nullptr) {
  const int t = lane & 3;
  uint32_t h1[4][4];  // A fragments of layer 2 (4 k steps)
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    uint32_t b[2];
    load_b(b, M.w1, kMlpInPad, 8 * j, 0, lane);
    mma_bf16_16816(d, a_in, b);
    const float bb0 = M.b1[8 * j + 2 * t], bb1 = M.b1[8 * j + 2 * t + 1];
    d[0] += bb0; d[1] += bb1; d[2] += bb0; d[3] += bb1;
    if (z1) {
#pragma unroll
      for (int e = 0; e < 4; ++e) z1[j][e] = d[e];
    }
    const uint32_t lo = pack_bf16x2(gelu(d[0]), gelu(d[1]));
    const uint32_t hi = pack_bf16x2(gelu(d[2]), gelu(d[3]));
    // tile j holds columns 8j..8j+7: k step j/2, low (j even) or high half
    if ((j & 1) == 0) { h1[j >> 1][0] = lo; h1[j >> 1][1] = hi; }
    else { h1[j >> 1][2] = lo; h1[j >> 1][3] = hi; }
  }
  float acc_lo = 0.f, acc_hi = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      uint32_t b[2];
      load_b(b, M.w2, kMlpH, 8 * j, 16 * ks, lane);
      mma_bf16_16816(d, h1[ks], b);
    }
    const int c0 = 8 * j + 2 * t;
    const float bb0 = M.b2[c0], bb1 = M.b2[c0 + 1];
    d[0] += bb0; d[1] += bb1; d[2] += bb0; d[3] += bb1;
    if (z2) {
#pragma unroll
      for (int e = 0; e < 4; ++e) z2[j][e] = d[e];
    }
    const float w0 = M.w3[c0], w1 = M.w3[c0 + 1];
    acc_lo = fmaf(gelu(d[0]), w0, fmaf(gelu(d[1]), w1, acc_lo));
    acc_hi = fmaf(gelu(d[2]), w0, fmaf(gelu(d[3]), w1, acc_hi));
  }
  // the four lanes of a quad hold disjoint columns of rows g and g+8
  acc_lo += __shfl_xor_sync(0xffffffffu, acc_lo, 1);
  acc_lo += __shfl_xor_sync(0xffffffffu, acc_lo, 2);
  acc_hi += __shfl_xor_sync(0xffffffffu, acc_hi, 1);
  acc_hi += __shfl_xor_sync(0xffffffffu, acc_hi, 2);
  y_lo = acc_lo + M.b3[0];
  y_hi = acc_hi + M.b3[0];
}

// A fragment of a 16-row tile of features stored row-major (stride 16 bf16)
// in shared memory.
__device__ __forceinline__ void load_a_rows16(uint32_t a[4], const __nv_bfloat16* s, int lane) {
  const int g = lane >> 2, t = lane & 3;
  a[0] = *reinterpret_cast<const uint32_t*>(s + g * 16 + 2 * t);
  a[1] = *reinterpret_cast<const uint32_t*>(s + (g + 8) * 16 + 2 * t);
  a[2] = *reinterpret_cast<const uint32_t*>(s + g * 16 + 2 * t + 8);
  a[3] = *reinterpret_cast<const uint32_t*>(s + (g + 8) * 16 + 2 * t + 8);
}

}  // namespace pbf
