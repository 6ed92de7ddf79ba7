// Fast-math gather kernels of the PBF step (exact_math = 0).
//
// Same stages, same neighbor lists, same results within the 1e-5 parity
// tolerance as the exact kernels, restructured for issue rate and memory-level
// parallelism on sm_100a:
//  - one rsqrt per pair: rinv = rsqrt(d^2), r = d^2*rinv; Poly6 uses h^2 - d^2
//    directly; Del_Spikey's r/(r + FLT_EPSILON) becomes r*rinv (both vanish at
//    r = 0; they differ by FLT_EPSILON/r relative);
//  - branch-free: clamping (h^2 - d^2) and (h - r) at 0 zeroes the pairs with
//    h < r < s, which stay in the lists because x* moves during the iterations;
//  - kernel constants (norms, 1/rho0, mass) folded on the host;
//  - GL = 4 or 8 lanes per particle (the launch shape the autotuner picks)
//    walk its row-major list together (see Group) and combine their partial
//    sums with shuffles.
// A particle sitting exactly on a neighbour (d^2 < 1e-16, the reference's
// nudge condition |r| < 1e-8, particles.h:303-305) falls back to the
// reference-ordered path for that particle.
#pragma once
#include "pbf_kernels.cuh"

namespace pbf {

// Constants of the fast path, derived from Dev on the host.
struct Fast {
  float h, h2, m_w0;     // h, h^2, m*Poly6(0)
  float m_poly;          // m * poly6 norm: rho = m_w0 + m_poly * sum (h^2-d^2)^3
  float lam_grad;        // -spikey_norm / rho0: grad C_j = lam_grad * (h-r)^2/r * r_vec
  float dp_scale;        // spikey_norm / rho0: dp = dp_scale * sum (l_p+l_q) (h-r)^2/r * r_vec
  float visc_poly;       // poly6 norm (W = visc_poly * (h^2-d^2)^3)
  float spikey;          // spikey norm
  float inv_rho0, lambda_eps, visc_c, vort_dt;  // vort_dt = vorticity_coef * dt
};

inline Fast make_fast(const Dev& d) {
  Fast f;
  f.h = d.h;
  f.h2 = d.h * d.h;
  f.m_w0 = d.m * d.W0;
  f.m_poly = d.m * d.poly6_norm;
  f.lam_grad = -d.spikey_norm / d.rho0;
  f.dp_scale = d.spikey_norm / d.rho0;
  f.visc_poly = d.poly6_norm;
  f.spikey = d.spikey_norm;
  f.inv_rho0 = d.inv_rho0;
  f.lambda_eps = d.lambda_eps;
  f.visc_c = d.visc_c;
  f.vort_dt = d.vort_eps * d.dt;
  return f;
}

// Lane groups: GL consecutive threads share one particle (GL = 4 or 8, the
// launch shape the autotuner picks per kernel family; kGL is the default).
// Lane l walks entries l, l + GL, ... of the particle's row-major list, so one
// warp-wide load touches GL consecutive entries of each of 32/GL lists, and
// the neighbours those entries name are mostly consecutive slots of one bin
// (coalesced gathers).  Partial sums are combined with shuffles.
constexpr int kGL = 8;

struct Group {
  int b;      // particle slot (0 for threads past the end, which walk nothing)
  int lane;   // 0 .. GL-1
  bool live;  // b < n
};

// Group of this thread in block-sized tile `tile` (grid-stride kernels walk
// several tiles per block).
template <int GL = kGL>
__device__ __forceinline__ Group group_at(int n, int tile) {
  const int gid = tile * blockDim.x + threadIdx.x;
  Group g;
  g.b = gid / GL;
  g.lane = gid % GL;
  g.live = g.b < n;
  if (!g.live) g.b = 0;
  return g;
}

template <int GL = kGL>
__device__ __forceinline__ Group group_of(int n) {
  return group_at<GL>(n, blockIdx.x);
}

// Tiles of blockDim.x threads covering n particles at GL lanes each.
template <int GL>
__device__ __forceinline__ int tiles_of(int n) {
  return (int)(((size_t)n * GL + blockDim.x - 1) / blockDim.x);
}

// Sum over the GL lanes of a group (every lane of the warp must call it).
template <int GL = kGL>
__device__ __forceinline__ float gsum(float v) {
#pragma unroll
  for (int o = GL / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, GL);
  return v;
}

template <int GL = kGL>
__device__ __forceinline__ int gor(int v) {
#pragma unroll
  for (int o = GL / 2; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o, GL);
  return v;
}

template <int GL = kGL>
__device__ __forceinline__ float gmin(float v) {
#pragma unroll
  for (int o = GL / 2; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o, GL));
  return v;
}

// Walk entries lane, lane + GL, ... of a list row, kB entries per batch:
// the batch's indices are loaded first, then its neighbour records, then the
// bodies run (predicated past the count), keeping 2*kB loads in flight.
constexpr int kB = 4;

template <int GL = kGL, class Body>
__device__ __forceinline__ void gwalk1(const int32_t* __restrict__ row, int c, int lane,
                                       const float4* __restrict__ a, Body&& body) {
  for (int k0 = lane; k0 < c; k0 += kB * GL) {
    int q[kB];
    float4 v[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int k = k0 + u * GL;
      q[u] = k < c ? __ldg(row + k) : -1;
    }
#pragma unroll
    for (int u = 0; u < kB; ++u)
      if (q[u] >= 0) v[u] = __ldg(a + q[u]);
#pragma unroll
    for (int u = 0; u < kB; ++u)
      if (q[u] >= 0) body(q[u], v[u]);
  }
}

// Two records per neighbour: batches of kB2 keep the register count (and so
// the occupancy) of the one-record walk (batches of 4 at 4 lanes measured
// slower: 64 registers).
constexpr int kB2 = 2;

template <int GL = kGL, class Body>
__device__ __forceinline__ void gwalk2(const int32_t* __restrict__ row, int c, int lane,
                                       const float4* __restrict__ a, const float4* __restrict__ bsrc,
                                       Body&& body) {
  constexpr int kB = kB2;
  for (int k0 = lane; k0 < c; k0 += kB * GL) {
    int q[kB];
    float4 va[kB], vb[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int k = k0 + u * GL;
      q[u] = k < c ? __ldg(row + k) : -1;
    }
#pragma unroll
    for (int u = 0; u < kB; ++u)
      if (q[u] >= 0) {
        va[u] = __ldg(a + q[u]);
        vb[u] = __ldg(bsrc + q[u]);
      }
#pragma unroll
    for (int u = 0; u < kB; ++u)
      if (q[u] >= 0) body(q[u], va[u], vb[u]);
  }
}

// (h - r)^2 / r for r < h, else 0 (the Del_Spikey magnitude over r, no norm).
__device__ __forceinline__ float spikey_over_r(const Fast& F, float d2) {
  const float rinv = rsqrtf(fmaxf(d2, 1e-30f));
  const float hr = fmaxf(fmaf(-d2, rinv, F.h), 0.0f);  // h - r
  return hr * hr * rinv;
}

__device__ __forceinline__ float poly_cube(const Fast& F, float d2) {
  const float a = fmaxf(F.h2 - d2, 0.0f);
  return a * a * a;
}

}  // namespace pbf
