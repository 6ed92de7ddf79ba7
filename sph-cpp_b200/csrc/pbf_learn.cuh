// Training and inference kernels of the learned warm start (see pbf_mlp.cuh).
//
// Training: the fused plain step records, per particle, the 12 features at its
// first Jacobi iteration and, as label, the sum of the lambdas the plain solver
// applied over its K iterations (delta-p is linear in lambda, so one delta-p
// with that sum approximates the K iterations).  k_mlp_grad_tc
// (pbf_train_tc.cuh) evaluates the network forward and backward on a batch
// drawn from that record, every GEMM on the tensor cores (BF16 operands, FP32
// accumulation); k_mlp_adam applies Adam to the FP32 master parameters;
// k_mlp_sync refreshes the BF16 operand copies.
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
// LOOP: the check sits in the graph's conditional loop and sets its handle;
// a check outside the loop is compiled without the call (a kernel that can
// set a conditional handle is one ncu cannot profile).
template <int THREADS, bool LOOP>
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
  if constexpr (LOOP) {
    if (loop.use) {
      // One more pass of the loop only while the step is not done and another
      // plain iteration is allowed; `loops` bounds the loop whatever the
      // residuals do.
      st->loops += 1u;
      const bool more = !st->done && st->iterations + 1u < (uint32_t)loop.iters && st->loops < (uint32_t)loop.iters;
      cudaGraphSetConditional(loop.cond, more ? 1u : 0u);
    }
  }
}

}  // namespace pbf
