// Training and inference kernels of the learned warm start (see pbf_mlp.cuh).
//
// Training: the fused plain step records, per particle, the 12 features at its
// first Jacobi iteration and, as label, the sum of the lambdas the plain solver
// applied over its K iterations (delta-p is linear in lambda, so one delta-p
// with that sum approximates the K iterations).  k_mlp_grad evaluates the
// network forward and backward on a batch drawn from that record, all GEMMs on
// the tensor cores (BF16 operands, FP32 accumulation); k_mlp_adam applies Adam
// to the FP32 master parameters; k_mlp_sync refreshes the BF16 operand copies.
#pragma once
#include "pbf_fast.cuh"
#include "pbf_mlp.cuh"

namespace pbf {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Generic A fragment of a row-major [m][k] bf16 matrix (stride ld).
__device__ __forceinline__ void load_a(uint32_t a[4], const __nv_bfloat16* s, int ld, int m0, int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  a[0] = *reinterpret_cast<const uint32_t*>(s + (m0 + g) * ld + k0 + 2 * t);
  a[1] = *reinterpret_cast<const uint32_t*>(s + (m0 + g + 8) * ld + k0 + 2 * t);
  a[2] = *reinterpret_cast<const uint32_t*>(s + (m0 + g) * ld + k0 + 2 * t + 8);
  a[3] = *reinterpret_cast<const uint32_t*>(s + (m0 + g + 8) * ld + k0 + 2 * t + 8);
}

// fp32 masters -> BF16 operands (W1 zero-padded to k = 16, W2 both ways).
__global__ void k_mlp_sync(const float* __restrict__ P, __nv_bfloat16* w1b, __nv_bfloat16* w2b,
                           __nv_bfloat16* w2tb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kMlpH * kMlpInPad) {
    const int n = i / kMlpInPad, k = i % kMlpInPad;
    w1b[i] = __float2bfloat16_rn(k < kMlpIn ? P[kOffW1 + n * kMlpIn + k] : 0.0f);
  }
  if (i < kMlpH * kMlpH) {
    const int n = i / kMlpH, k = i % kMlpH;
    const __nv_bfloat16 w = __float2bfloat16_rn(P[kOffW2 + n * kMlpH + k]);
    w2b[i] = w;
    w2tb[k * kMlpH + n] = w;
  }
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8); c1, c2 are the bias corrections
// 1/(1-beta^t) of this step.
__global__ void k_mlp_adam(float* P, const float* __restrict__ G, float* m, float* v, int np, float lr, float c1,
                           float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const float g = G[i];
  const float mi = 0.9f * m[i] + 0.1f * g;
  const float vi = 0.999f * v[i] + 0.001f * g * g;
  m[i] = mi;
  v[i] = vi;
  P[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
}

// Row of sample i: drawn from n_data rows by a counter-based hash when
// SAMPLE, else row i itself.
template <bool SAMPLE>
__device__ __forceinline__ int sample_row(uint64_t seed, int i, int n_data) {
  if (!SAMPLE) return i;
  return (int)(mix64(seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(i + 1))) % (uint64_t)n_data);
}

// Sum of v over the 8 lanes sharing t = lane % 4 (the row groups of a tile).
__device__ __forceinline__ float sum_over_g(float v) {
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  v += __shfl_xor_sync(0xffffffffu, v, 8);
  v += __shfl_xor_sync(0xffffffffu, v, 16);
  return v;
}

constexpr int kGradRows = 64;  // samples per block: 4 warps x 16 rows

// Gradient of L = mean over the batch of (y - target)^2, accumulated into
// grad (fp32, canonical order) with atomics; L into *loss.
// NORMALIZE: features are raw and normalised here (else already normalised).
// SAMPLE: rows drawn from the n_data recorded rows (else rows 0..batch-1);
// targets = labels * inv_label_scale.
template <bool NORMALIZE, bool SAMPLE>
__global__ void __launch_bounds__(128) k_mlp_grad(MlpDev M, const float* __restrict__ feats,
                                                  const float* __restrict__ labels, int n_data, int batch,
                                                  uint64_t seed, float inv_label_scale, float* grad, float* loss) {
  __shared__ __align__(16) __nv_bfloat16 sX[kGradRows * kMlpInPad];   // X [row][k]
  __shared__ __align__(16) __nv_bfloat16 sXT[kMlpInPad * kGradRows];  // X^T [k][row]
  __shared__ __align__(16) __nv_bfloat16 sH1T[kMlpH * kGradRows];     // H1^T [k][row]
  __shared__ __align__(16) __nv_bfloat16 sD2T[kMlpH * kGradRows];     // dZ2^T [n][row]
  __shared__ __align__(16) __nv_bfloat16 sD1T[kMlpH * kGradRows];     // dZ1^T [n][row]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int base = blockIdx.x * kGradRows;
  for (int e = threadIdx.x; e < kGradRows * kMlpInPad; e += blockDim.x) {
    const int r = e / kMlpInPad, k = e % kMlpInPad;
    const int i = base + r;
    float f = 0.0f;
    if (i < batch && k < kMlpIn) {
      const float x = feats[(size_t)sample_row<SAMPLE>(seed, i, n_data) * kMlpIn + k];
      f = NORMALIZE ? (x - M.feat_mean[k]) * M.feat_inv_std[k] : x;
    }
    const __nv_bfloat16 b = __float2bfloat16_rn(f);
    sX[r * kMlpInPad + k] = b;
    sXT[k * kGradRows + r] = b;
  }
  __syncthreads();

  // forward, keeping the pre-activations
  uint32_t a[4];
  load_a(a, sX, kMlpInPad, warp * 16, 0, lane);
  float z1[8][4], z2[8][4], y_lo, y_hi;
  mlp_forward16(M, a, lane, y_lo, y_hi, z1, z2);
  const int r_lo = warp * 16 + g, r_hi = r_lo + 8;
  const bool ok_lo = base + r_lo < batch, ok_hi = base + r_hi < batch;
  const float t_lo = ok_lo ? labels[sample_row<SAMPLE>(seed, base + r_lo, n_data)] * inv_label_scale : 0.f;
  const float t_hi = ok_hi ? labels[sample_row<SAMPLE>(seed, base + r_hi, n_data)] * inv_label_scale : 0.f;
  const float inv_b = 1.0f / (float)batch;
  const float e_lo = ok_lo ? y_lo - t_lo : 0.f, e_hi = ok_hi ? y_hi - t_hi : 0.f;
  const float dy_lo = 2.0f * e_lo * inv_b, dy_hi = 2.0f * e_hi * inv_b;
  {
    float l = t == 0 ? (e_lo * e_lo + e_hi * e_hi) * inv_b : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    float db3 = t == 0 ? dy_lo + dy_hi : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) db3 += __shfl_xor_sync(0xffffffffu, db3, o);
    if (lane == 0) {
      atomicAdd(loss, l);
      atomicAdd(grad + kOffB3, db3);
    }
  }
  // layer 3 and GELU of layer 2: dW3, dZ2 (in place of z2), db2
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c0 = 8 * j + 2 * t;
    const float gw0 = sum_over_g(gelu(z2[j][0]) * dy_lo + gelu(z2[j][2]) * dy_hi);
    const float gw1 = sum_over_g(gelu(z2[j][1]) * dy_lo + gelu(z2[j][3]) * dy_hi);
    const float w0 = M.w3[c0], w1 = M.w3[c0 + 1];
    z2[j][0] = dy_lo * w0 * gelu_grad(z2[j][0]);
    z2[j][1] = dy_lo * w1 * gelu_grad(z2[j][1]);
    z2[j][2] = dy_hi * w0 * gelu_grad(z2[j][2]);
    z2[j][3] = dy_hi * w1 * gelu_grad(z2[j][3]);
    const float gb0 = sum_over_g(z2[j][0] + z2[j][2]);
    const float gb1 = sum_over_g(z2[j][1] + z2[j][3]);
    if (g == 0) {
      atomicAdd(grad + kOffW3 + c0, gw0);
      atomicAdd(grad + kOffW3 + c0 + 1, gw1);
      atomicAdd(grad + kOffB2 + c0, gb0);
      atomicAdd(grad + kOffB2 + c0 + 1, gb1);
    }
    sD2T[c0 * kGradRows + r_lo] = __float2bfloat16_rn(z2[j][0]);
    sD2T[(c0 + 1) * kGradRows + r_lo] = __float2bfloat16_rn(z2[j][1]);
    sD2T[c0 * kGradRows + r_hi] = __float2bfloat16_rn(z2[j][2]);
    sD2T[(c0 + 1) * kGradRows + r_hi] = __float2bfloat16_rn(z2[j][3]);
    sH1T[c0 * kGradRows + r_lo] = __float2bfloat16_rn(gelu(z1[j][0]));
    sH1T[(c0 + 1) * kGradRows + r_lo] = __float2bfloat16_rn(gelu(z1[j][1]));
    sH1T[c0 * kGradRows + r_hi] = __float2bfloat16_rn(gelu(z1[j][2]));
    sH1T[(c0 + 1) * kGradRows + r_hi] = __float2bfloat16_rn(gelu(z1[j][3]));
  }
  // dH1 = dZ2 W2 on the tensor cores (A = dZ2 repacked, B = W2^T k-major), then dZ1
  uint32_t ad[4][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint32_t lo = pack_bf16x2(z2[j][0], z2[j][1]);
    const uint32_t hi = pack_bf16x2(z2[j][2], z2[j][3]);
    if ((j & 1) == 0) { ad[j >> 1][0] = lo; ad[j >> 1][1] = hi; }
    else { ad[j >> 1][2] = lo; ad[j >> 1][3] = hi; }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      uint32_t b[2];
      load_b(b, M.w2t, kMlpH, 8 * j, 16 * ks, lane);
      mma_bf16_16816(d, ad[ks], b);
    }
    const int c0 = 8 * j + 2 * t;
    const float d0 = d[0] * gelu_grad(z1[j][0]), d1 = d[1] * gelu_grad(z1[j][1]);
    const float d2 = d[2] * gelu_grad(z1[j][2]), d3 = d[3] * gelu_grad(z1[j][3]);
    const float gb0 = sum_over_g(d0 + d2), gb1 = sum_over_g(d1 + d3);
    if (g == 0) {
      atomicAdd(grad + kOffB1 + c0, gb0);
      atomicAdd(grad + kOffB1 + c0 + 1, gb1);
    }
    sD1T[c0 * kGradRows + r_lo] = __float2bfloat16_rn(d0);
    sD1T[(c0 + 1) * kGradRows + r_lo] = __float2bfloat16_rn(d1);
    sD1T[c0 * kGradRows + r_hi] = __float2bfloat16_rn(d2);
    sD1T[(c0 + 1) * kGradRows + r_hi] = __float2bfloat16_rn(d3);
  }
  __syncthreads();
  // dW2[n][k] = sum_rows dZ2[row][n] H1[row][k]: warp w owns n = 16w..16w+15
  {
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
#pragma unroll
    for (int ks = 0; ks < kGradRows / 16; ++ks) {
      uint32_t af[4];
      load_a(af, sD2T, kGradRows, 16 * warp, 16 * ks, lane);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        uint32_t b[2];
        load_b(b, sH1T, kGradRows, 8 * j, 16 * ks, lane);
        mma_bf16_16816(acc[j], af, b);
      }
    }
    const int n_lo = 16 * warp + g;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k0 = 8 * j + 2 * t;
      atomicAdd(grad + kOffW2 + n_lo * kMlpH + k0, acc[j][0]);
      atomicAdd(grad + kOffW2 + n_lo * kMlpH + k0 + 1, acc[j][1]);
      atomicAdd(grad + kOffW2 + (n_lo + 8) * kMlpH + k0, acc[j][2]);
      atomicAdd(grad + kOffW2 + (n_lo + 8) * kMlpH + k0 + 1, acc[j][3]);
    }
  }
  // dW1[n][k] = sum_rows dZ1[row][n] X[row][k] (k < 12)
  {
    float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
    for (int ks = 0; ks < kGradRows / 16; ++ks) {
      uint32_t af[4];
      load_a(af, sD1T, kGradRows, 16 * warp, 16 * ks, lane);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        uint32_t b[2];
        load_b(b, sXT, kGradRows, 8 * j, 16 * ks, lane);
        mma_bf16_16816(acc[j], af, b);
      }
    }
    const int n_lo = 16 * warp + g;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int k0 = 8 * j + 2 * t;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int n = n_lo + (e >= 2 ? 8 : 0), k = k0 + (e & 1);
        if (k < kMlpIn) atomicAdd(grad + kOffW1 + n * kMlpIn + k, acc[j][e]);
      }
    }
  }
}

// ---- features and the residual-checked solve ----

// Raw features of a particle at its first Jacobi iteration (order documented
// in pbf.h).  sc_nb = sum_j |grad C_j|^2, g2 = |grad C_i|^2.
__device__ __forceinline__ void raw_features(const Dev& P, const Region& R, const Fast& F, float f[kMlpIn], int c,
                                             float rho, float sc_nb, float g2, int nh, float lamprev, float4 v,
                                             float4 xp) {
  const float rel = rho * F.inv_rho0 - 1.0f;
  const float C = fmaxf(rel, 0.0f);
  const float S = sc_nb + g2;
  const float inv_h = 1.0f / P.h;
  f[0] = (float)c * (1.0f / 64.0f);
  f[1] = C;
  f[2] = rel;
  f[3] = S;
  f[4] = -C / (S + F.lambda_eps);
  f[5] = lamprev;
  f[6] = S > 0.0f ? g2 / S : 0.0f;
  f[7] = c > 0 ? (float)nh / (float)c : 0.0f;
  f[8] = v.y * P.dt * inv_h;
  f[9] = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z) * P.dt * inv_h;
  f[10] = fminf((xp.y - R.bmin[1]) * inv_h, 4.0f);
  float wall = fminf(fminf(xp.x - R.bmin[0], R.bmax[0] - xp.x), fminf(xp.y - R.bmin[1], R.bmax[1] - xp.y));
  wall = fminf(wall, fminf(xp.z - R.bmin[2], R.bmax[2] - xp.z));
  f[11] = fminf(wall * inv_h, 4.0f);
}

// Solver state of the learned warm start, reset each step.
struct SolveState {
  double residual;      // mean clamped density error at the last check
  uint32_t done;        // residual at or below the tolerance: the rest of the step's iterations skip
  uint32_t iterations;  // Jacobi iterations applied this step
  uint32_t ticket;      // blocks of the running check that have written their partial sum
  uint32_t loops;       // checks run inside the graph's conditional loop this step
};

// The graph's conditional loop around the learned solver's plain iterations
// (a WHILE node whose body is one residual check and one position update;
// the check ends the loop).  use = 0: no loop (eager launches, or the check
// after the loop).
struct SolveLoop {
  cudaGraphConditionalHandle cond;
  int use;
  int iters;  // max_iterations: the loop runs at most iters - 1 times
};

// Sum of v over the block (every thread calls it; blockDim.x a multiple of 32,
// at most THREADS), written by thread 0 to *out.  Warp sums in float, the
// warps' sums added in double in warp order: the same inputs give the same
// bits on every run.
template <int THREADS>
__device__ __forceinline__ void block_partial(float v, double* out) {
  __shared__ float warp_sum[THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    const int warps = (int)(blockDim.x >> 5);
    for (int w = 0; w < warps; ++w) s += (double)warp_sum[w];
    *out = s;
  }
}

// The end of a residual check (every thread of every block calls it, after
// block_partial): the last block to finish adds the grid's partial sums in a
// fixed order (so the decision is the same on every run) and either stops the
// step's iterations (mean error at or below tol) or allows one more (the final
// check of a step only records the residual).
template <int THREADS>
__device__ __forceinline__ void decide_if_last(SolveState* st, const double* partials, int n, float tol,
                                               int final_check, SolveLoop loop) {
  __shared__ unsigned last;
  __shared__ double red[THREADS];
  if (threadIdx.x == 0) {
    __threadfence();  // this block's partial before its ticket
    last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1u;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double s = 0.0;
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) s += __ldcg(partials + i);
  red[threadIdx.x] = s;
  __syncthreads();
  for (unsigned o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double mean = red[0] / (double)(n > 0 ? n : 1);
  st->residual = mean;
  st->ticket = 0u;
  if (mean <= (double)tol) st->done = 1u;
  else if (!final_check) st->iterations += 1u;
  if (loop.use) {
    // One more pass of the loop only while the step is not done and another
    // plain iteration is allowed; `loops` bounds the loop whatever the
    // residuals do.
    st->loops += 1u;
    const bool more = !st->done && st->iterations + 1u < (uint32_t)loop.iters && st->loops < (uint32_t)loop.iters;
    cudaGraphSetConditional(loop.cond, more ? 1u : 0u);
  }
}

}  // namespace pbf
