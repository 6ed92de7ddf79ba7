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
//  - GL = 2, 4 or 8 lanes per particle (the launch shape the autotuner picks)
//    walk its warp-tiled, padded list together (see Group, gwalk1) and
//    combine their partial sums with shuffles.
// A particle sitting exactly on a neighbour (d^2 < 1e-16, the reference's
// nudge condition |r| < 1e-8, particles.h:303-305) falls back to the
// reference-ordered path for that particle.
#pragma once
#include <cuda_fp16.h>
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

// Lane groups: GL consecutive threads share one particle (GL = 2, 4 or 8, the
// launch shape the autotuner picks per kernel family; kGL is the default).
// Lane l walks its share of every batch of the particle's list (gwalk1,
// gwalk2); a warp-wide index load reads the same chunk row of 32/GL
// consecutive particles' lists, contiguous in the warp-tiled layout.  Partial
// sums are combined with shuffles.
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

// Vector v of a particle's list (entries 4v..4v+3, or 2v, 2v+1 for the 8-byte
// vectors) in the warp-tiled layout (list_base, list_off): the row pointer is
// the particle's first entry, its 8-entry chunks 128 entries apart.
__device__ __forceinline__ int vec4_at(int v) { return (v >> 1) * (kListTile * kListChunk / 4) + (v & 1); }
__device__ __forceinline__ int vec2_at(int v) { return (v >> 2) * (kListTile * kListChunk / 2) + (v & 3); }
// A batch of a walk covers whole chunks when GL is even (4*GL entries per
// batch) or a multiple of 4 (2*GL entries): batch t starts t * 16 * GL
// vectors in (its 4*GL or 2*GL entries span GL/2 or GL/4 chunk rows), and
// lane l's vector sits at vec4_at(l) / vec2_at(l) from there.
constexpr int kBatchVecs = kListTile * kListChunk / 8;  // x GL: vectors per batch

// Loads of the walks.  The read-only path (__ldg, ld.global.nc) for arrays
// no thread writes during the launch; COH: plain loads (ld.global, cached in
// L1), for the persistent step, one launch whose passes write what later
// passes read.  A pass there reads only after an acquire at GPU scope, which
// drops the SM's L1 lines that other SMs have written since; the read-only
// path promises no such thing.
template <bool COH, class T>
__device__ __forceinline__ T ldw(const T* p) {
  if constexpr (COH)
    return *p;
  else
    return __ldg(p);
}

// The last batch: entries of vector v (entries 4v..4v+3, or 2v, 2v+1) at or
// past the count c name `dummy`.
__device__ __forceinline__ int4 tail4(int4 q, int v, int c, int dummy) {
  const int e = 4 * v;
  q.x = e < c ? q.x : dummy;
  q.y = e + 1 < c ? q.y : dummy;
  q.z = e + 2 < c ? q.z : dummy;
  q.w = e + 3 < c ? q.w : dummy;
  return q;
}
__device__ __forceinline__ int2 tail2(int2 q, int v, int c, int dummy) {
  const int e = 2 * v;
  q.x = e < c ? q.x : dummy;
  q.y = e + 1 < c ? q.y : dummy;
  return q;
}

// Walk a list row: lane l of the group takes four entries of every 4*GL-entry
// batch (the 16-byte vector vec4_at), one index load, then its four neighbour records
// (four independent loads in flight), then the four bodies.  Rows are padded
// to a multiple of 32 entries, so every batch reads whole vectors inside the
// row; entries of the last batch past the count are replaced by `dummy`, a
// slot whose every term is zero.  PF: the next batch's index vector is loaded
// before this batch's records (the lists stream from DRAM; the prefetch takes
// one DRAM round trip per batch off the index -> record chain).  It is set
// where it measured faster (the final XSPH pass); elsewhere it measured
// slower (Δp too, since the warp-tiled lists).
template <int GL = kGL, bool PF = false, bool COH = false, class Body>
__device__ __forceinline__ void gwalk1(const int32_t* __restrict__ row, int c, int dummy, int lane,
                                       const float4* __restrict__ a, Body&& body) {
  static_assert(GL % 2 == 0, "a batch covers whole chunks");
  const int4* r4 = reinterpret_cast<const int4*>(row);
  const int l0 = vec4_at(lane);
  if constexpr (PF) {
    const int batches = (c + 4 * GL - 1) / (4 * GL);
    if (batches == 0) return;
    int4 next = ldw<COH>(r4 + l0);
    for (int t = 0; t < batches; ++t) {
      int4 q = next;
      if (t + 1 < batches) next = ldw<COH>(r4 + (l0 + (t + 1) * kBatchVecs * GL));
      if (t + 1 == batches) q = tail4(q, t * GL + lane, c, dummy);
      const float4 v0 = ldw<COH>(a + q.x), v1 = ldw<COH>(a + q.y);
      const float4 v2 = ldw<COH>(a + q.z), v3 = ldw<COH>(a + q.w);
      body(q.x, v0);
      body(q.y, v1);
      body(q.z, v2);
      body(q.w, v3);
    }
  } else {
    const int full = c / (4 * GL);
    int t = 0;
    for (; t < full; ++t) {
      const int4 q = ldw<COH>(r4 + (l0 + t * kBatchVecs * GL));
      const float4 v0 = ldw<COH>(a + q.x), v1 = ldw<COH>(a + q.y);
      const float4 v2 = ldw<COH>(a + q.z), v3 = ldw<COH>(a + q.w);
      body(q.x, v0);
      body(q.y, v1);
      body(q.z, v2);
      body(q.w, v3);
    }
    if (t * 4 * GL < c) {
      const int4 q = tail4(ldw<COH>(r4 + (l0 + t * kBatchVecs * GL)), t * GL + lane, c, dummy);
      const float4 v0 = ldw<COH>(a + q.x), v1 = ldw<COH>(a + q.y);
      const float4 v2 = ldw<COH>(a + q.z), v3 = ldw<COH>(a + q.w);
      body(q.x, v0);
      body(q.y, v1);
      body(q.z, v2);
      body(q.w, v3);
    }
  }
}

// Two records per neighbour: entries 2l, 2l+1 of every 2*GL-entry batch (an
// 8-byte index load), so that four records are in flight per lane, as in the
// one-record walk; PF as there.
template <int GL = kGL, bool PF = false, bool COH = false, class Body>
__device__ __forceinline__ void gwalk2(const int32_t* __restrict__ row, int c, int dummy, int lane,
                                       const float4* __restrict__ a, const float4* __restrict__ bsrc,
                                       Body&& body) {
  const int2* r2 = reinterpret_cast<const int2*>(row);
  // vector of batch t (whole chunk rows when GL is a multiple of 4)
  auto at = [&](int t) { return GL % 4 == 0 ? t * kBatchVecs * GL + vec2_at(lane) : vec2_at(t * GL + lane); };
  if constexpr (PF) {
    const int batches = (c + 2 * GL - 1) / (2 * GL);
    if (batches == 0) return;
    int2 next = ldw<COH>(r2 + at(0));
    for (int t = 0; t < batches; ++t) {
      int2 q = next;
      if (t + 1 < batches) next = ldw<COH>(r2 + at(t + 1));
      if (t + 1 == batches) q = tail2(q, t * GL + lane, c, dummy);
      const float4 a0 = ldw<COH>(a + q.x), b0 = ldw<COH>(bsrc + q.x);
      const float4 a1 = ldw<COH>(a + q.y), b1 = ldw<COH>(bsrc + q.y);
      body(q.x, a0, b0);
      body(q.y, a1, b1);
    }
  } else {
    const int full = c / (2 * GL);
    int t = 0;
    for (; t < full; ++t) {
      const int2 q = ldw<COH>(r2 + at(t));
      const float4 a0 = ldw<COH>(a + q.x), b0 = ldw<COH>(bsrc + q.x);
      const float4 a1 = ldw<COH>(a + q.y), b1 = ldw<COH>(bsrc + q.y);
      body(q.x, a0, b0);
      body(q.y, a1, b1);
    }
    if (t * 2 * GL < c) {
      const int2 q = tail2(ldw<COH>(r2 + at(t)), t * GL + lane, c, dummy);
      const float4 a0 = ldw<COH>(a + q.x), b0 = ldw<COH>(bsrc + q.x);
      const float4 a1 = ldw<COH>(a + q.y), b1 = ldw<COH>(bsrc + q.y);
      body(q.x, a0, b0);
      body(q.y, a1, b1);
    }
  }
}

// The XSPH passes' weights W(r)/rho_q per list entry: both viscosity passes
// weigh a neighbour's velocity by the same value (x* and the densities do not
// change between them), so the first stores it beside its list entry (the
// same warp-tiled layout, `wrow` = the weight row of the particle's list row)
// and the final pass reads it as a coalesced stream instead of gathering the
// neighbour's x* (one scattered record per entry instead of two).  Stored
// in half precision (2 bytes per entry, the final pass's weight within 2^-11
// of the first pass's): half the weight stream's bytes, within the fast
// path's tolerances.
// gwalk2 that also stores body's return value per entry:
template <int GL = kGL, bool COH = false, class Body>
__device__ __forceinline__ void gwalk2w(const int32_t* __restrict__ row, __half* wrow, int c, int dummy, int lane,
                                        const float4* __restrict__ a, const float4* __restrict__ bsrc, Body&& body) {
  const int2* r2 = reinterpret_cast<const int2*>(row);
  __half2* w2 = reinterpret_cast<__half2*>(wrow);
  auto at = [&](int t) { return GL % 4 == 0 ? t * kBatchVecs * GL + vec2_at(lane) : vec2_at(t * GL + lane); };
  auto two = [&](int t, int2 q) {
    const float4 a0 = ldw<COH>(a + q.x), b0 = ldw<COH>(bsrc + q.x);
    const float4 a1 = ldw<COH>(a + q.y), b1 = ldw<COH>(bsrc + q.y);
    const float w0 = body(q.x, a0, b0);
    const float w1 = body(q.y, a1, b1);
    w2[at(t)] = __floats2half2_rn(w0, w1);
  };
  const int full = c / (2 * GL);
  int t = 0;
  for (; t < full; ++t) two(t, ldw<COH>(r2 + at(t)));
  if (t * 2 * GL < c) two(t, tail2(ldw<COH>(r2 + at(t)), t * GL + lane, c, dummy));
}

// The final pass's walk: entry q with its stored weight w and one record
// (entries past the count: the dummy record, weight 0); PF as gwalk1.
template <int GL = kGL, bool PF = false, bool COH = false, class Body>
__device__ __forceinline__ void gwalkw(const int32_t* __restrict__ row, const __half* __restrict__ wrow, int c,
                                       int dummy, int lane, const float4* __restrict__ bsrc, Body&& body) {
  const int2* r2 = reinterpret_cast<const int2*>(row);
  const __half2* w2 = reinterpret_cast<const __half2*>(wrow);
  auto at = [&](int t) { return GL % 4 == 0 ? t * kBatchVecs * GL + vec2_at(lane) : vec2_at(t * GL + lane); };
  auto two = [&](int2 q, float2 w) {
    const float4 b0 = ldw<COH>(bsrc + q.x), b1 = ldw<COH>(bsrc + q.y);
    body(q.x, w.x, b0);
    body(q.y, w.y, b1);
  };
  auto tail = [&](int t, int2& q, float2& w) {
    const int e = 2 * (t * GL + lane);
    if (e >= c) { q.x = dummy; w.x = 0.0f; }
    if (e + 1 >= c) { q.y = dummy; w.y = 0.0f; }
  };
  if constexpr (PF) {
    const int batches = (c + 2 * GL - 1) / (2 * GL);
    if (batches == 0) return;
    int2 next = ldw<COH>(r2 + at(0));
    __half2 wnext = ldw<COH>(w2 + at(0));
    for (int t = 0; t < batches; ++t) {
      int2 q = next;
      float2 w = __half22float2(wnext);
      if (t + 1 < batches) {
        next = ldw<COH>(r2 + at(t + 1));
        wnext = ldw<COH>(w2 + at(t + 1));
      }
      if (t + 1 == batches) tail(t, q, w);
      two(q, w);
    }
  } else {
    const int full = c / (2 * GL);
    int t = 0;
    for (; t < full; ++t) two(ldw<COH>(r2 + at(t)), __half22float2(ldw<COH>(w2 + at(t))));
    if (t * 2 * GL < c) {
      int2 q = ldw<COH>(r2 + at(t));
      float2 w = __half22float2(ldw<COH>(w2 + at(t)));
      tail(t, q, w);
      two(q, w);
    }
  }
}

// ---- staged walks: the tile's neighbour records in shared memory ----
// The list fill writes, beside each int32 list, a 16-bit list of indices into
// the tile's staging area (the neighbour bins of a 32-particle tile, copied to
// shared memory by the gather kernel; index `dummy` = the zero-contribution
// record past the staged ones).  Lane l of the group takes entries 8l..8l+7 of
// every 8*GL-entry batch (one 16-byte load), in two halves of four records.
__device__ __forceinline__ uint32_t lo16(uint32_t w) { return w & 0xffffu; }
__device__ __forceinline__ uint32_t hi16(uint32_t w) { return w >> 16; }

template <class Body>
__device__ __forceinline__ void stage_quad(const float4* stage, uint32_t w0, uint32_t w1, Body&& body) {
  const int i0 = (int)lo16(w0), i1 = (int)hi16(w0), i2 = (int)lo16(w1), i3 = (int)hi16(w1);
  const float4 v0 = stage[i0], v1 = stage[i1], v2 = stage[i2], v3 = stage[i3];
  body(i0, v0);
  body(i1, v1);
  body(i2, v2);
  body(i3, v3);
}

// Entries e and e+1 (the two halves of `word`): those at or past c name the dummy.
__device__ __forceinline__ uint32_t stage_fix(uint32_t word, int e, int c, uint32_t dummy) {
  const uint32_t lo = e < c ? lo16(word) : dummy;
  const uint32_t hi = e + 1 < c ? hi16(word) : dummy;
  return lo | (hi << 16);
}

// Entries e..e+7 of a 16-byte load (little-endian: w.x holds e, e+1).
__device__ __forceinline__ uint4 stage_tail(uint4 w, int e, int c, uint32_t dummy) {
  return make_uint4(stage_fix(w.x, e, c, dummy), stage_fix(w.y, e + 2, c, dummy), stage_fix(w.z, e + 4, c, dummy),
                    stage_fix(w.w, e + 6, c, dummy));
}

template <int GL = kGL, class Body>
__device__ __forceinline__ void swalk1(const uint16_t* __restrict__ row16, int c, int dummy, int lane,
                                       const float4* stage, Body&& body) {
  const uint4* r4 = reinterpret_cast<const uint4*>(row16);
  const int batches = (c + 8 * GL - 1) / (8 * GL);
  for (int t = 0; t < batches; ++t) {
    uint4 w = __ldg(r4 + t * GL + lane);
    if (t == batches - 1) w = stage_tail(w, t * 8 * GL + 8 * lane, c, (uint32_t)dummy);
    stage_quad(stage, w.x, w.y, body);
    stage_quad(stage, w.z, w.w, body);
  }
}

// Two staged records per neighbour (a, b staged at the same index).
template <int GL = kGL, class Body>
__device__ __forceinline__ void swalk2(const uint16_t* __restrict__ row16, int c, int dummy, int lane,
                                       const float4* sa, const float4* sb, Body&& body) {
  const uint4* r4 = reinterpret_cast<const uint4*>(row16);
  const int batches = (c + 8 * GL - 1) / (8 * GL);
  for (int t = 0; t < batches; ++t) {
    uint4 w = __ldg(r4 + t * GL + lane);
    if (t == batches - 1) w = stage_tail(w, t * 8 * GL + 8 * lane, c, (uint32_t)dummy);
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i0 = (int)lo16(ws[k]), i1 = (int)hi16(ws[k]);
      const float4 a0 = sa[i0], b0 = sb[i0], a1 = sa[i1], b1 = sb[i1];
      body(i0, a0, b0);
      body(i1, a1, b1);
    }
  }
}

// One walk for both sources: staged (shared memory, 16-bit list) or direct.
template <int GL, bool STAGED, bool PF = false, bool COH = false, class Body>
__device__ __forceinline__ void walk1(const int32_t* row, const uint16_t* row16, int c, int dummy, int lane,
                                      const float4* src, Body&& body) {
  if (STAGED)
    swalk1<GL>(row16, c, dummy, lane, src, body);
  else
    gwalk1<GL, PF, COH>(row, c, dummy, lane, src, body);
}

template <int GL, bool STAGED, bool PF = false, bool COH = false, class Body>
__device__ __forceinline__ void walk2(const int32_t* row, const uint16_t* row16, int c, int dummy, int lane,
                                      const float4* sa, const float4* sb, Body&& body) {
  if (STAGED)
    swalk2<GL>(row16, c, dummy, lane, sa, sb, body);
  else
    gwalk2<GL, PF, COH>(row, c, dummy, lane, sa, sb, body);
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
