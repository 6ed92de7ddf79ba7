// Per-particle MLP of the learned warm start: 12 -> 64 -> 64 -> 1, GELU
// (erf form), BF16 weights and activations, FP32 accumulation.  Its layout
// constants, the device view of its parameters and the activation functions;
// the tensor-core kernels are in pbf_mlp_tc.cuh (inference) and
// pbf_train_tc.cuh (training).
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

}  // namespace pbf
