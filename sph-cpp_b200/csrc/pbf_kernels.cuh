// Device-side math of the PBF step for sm_100a.
//
// Two evaluation policies share every kernel:
//   X = true  ("exact"): the reference's operation order with IEEE-rounded
//             __fadd_rn/__fmul_rn/__fdiv_rn/__fsqrt_rn, never contracted to FMA,
//             so results are bit-identical to the reference's gcc build
//             (x86-64, no FMA) on the same inputs and neighbor lists.
//   X = false ("fast"): FMA, reciprocal multiplies and rsqrt in the physics
//             gathers; results within the 1e-5 parity tolerance.
// The parts that decide neighbor sets (predict, boundary clamp, bin hash, the
// distance test) are always exact, so neighbor lists are bit-identical in both.
#pragma once
#include <cfloat>
#include <cstdint>

namespace pbf {

// Neighbour lists in warp tiles.  The lists of kListTile consecutive sorted
// slots interleave in chunks of kListChunk entries: entry j of slot b is at
//   (b / 16) * 16 * stride + (j / 8) * 128 + (b % 16) * 8 + j % 8
// (stride = the row length, a multiple of 32 entries).  A particle's chunk is
// one 32-byte sector, and the same chunk of 16 consecutive particles is 512
// contiguous bytes, so a warp of a gather that reads one chunk row of its
// particles' lists touches 4 cache lines, where row-major lists put each
// particle's chunk on a line of its own (one L1 wavefront per line).  The
// list buffer holds whole tiles: capacity rounded up to kListTile slots.
constexpr int kListTile = 16, kListChunk = 8;  // list_off's shift is log2(kListChunk)

__host__ __device__ inline size_t list_base(size_t b, size_t stride) {
  return (b / kListTile) * kListTile * stride + (b % kListTile) * kListChunk;
}
__host__ __device__ inline int list_off(int j) {
  return (j >> 3) * (kListTile * kListChunk) + (j & (kListChunk - 1));
}
__host__ __device__ inline size_t list_at(size_t b, size_t stride, int j) { return list_base(b, stride) + list_off(j); }
__host__ __device__ inline size_t list_entries(size_t capacity, size_t stride) {
  return (capacity + kListTile - 1) / kListTile * kListTile * stride;
}

// Box and bin grid of one scene.  A context advances one scene (the box and
// grid of Dev itself) or a batch of independent scenes, each with its own box
// and grid; the bin keys of a batch's scene i start at key0, so the sort by
// key keeps every scene's particles in one slot range, [first[i],
// first[i+1]), in every order the step uses.
struct Region {
  float bmin[3], bmax[3];
  int dimx, dimy, dimz;
  uint32_t key0;
};

// Per-launch constant block (kernel argument, < 4 KB).
struct Dev {
  float dt, gdt;  // time step; g*dt rounded in float (particles.h:264-268)
  float h, s, s2; // smoothing radius, bin spacing, s*s (neighbors.h:198)
  float m, rho0, inv_rho0, neg_inv_rho0;  // (Real)1/rho0, (Real)-1/rho0 (particles.h:332,356)
  float W0;       // Poly6(0) (particles.h:294)
  float poly6_norm, spikey_norm, cspline_norm;  // kernels.h:62,160,218 (double -> float)
  float lambda_eps, visc_c, vort_eps, gamma;
  float bmin[3], bmax[3], mc[3];
  float mr, mr2;  // mover radius and radius*radius in float (particles.h:515-519)
  float scorr_k, scorr_n, inv_wdq;
  double vthr;    // 0.000001 * max_speed, compared in double (particles.h:380)
  double h_eps;   // smoothing_radius * 0.000001 in double (particles.h:420)
  float skip_eps; // margin of the conservative bin skip in the list fill
  int dimx, dimy, dimz, nbins, cap;
  // batch of scenes (nscenes > 0): per-scene regions and first slots
  // (nscenes + 1 entries); nscenes = 0 is the single scene of the fields above
  const Region* scenes;
  const uint32_t* scene_first;
  int nscenes;
  // span of a per-stage call ([0, span_end) in reference index space, the
  // multi-rank driver's resident span): a stage updates the particles whose
  // reference index (span_orig of the slot) is below span_end and leaves the
  // others (halo particles) as they are; span_end = 0xffffffff is every particle
  const uint32_t* span_orig;
  uint32_t span_end;
};

// Whether the particle in home slot `i` is inside the stage's span.
__device__ __forceinline__ bool in_span(const Dev& P, int i) {
  return P.span_end == 0xffffffffu || __ldg(P.span_orig + i) < P.span_end;
}

// The region of the particle in `slot` (any order the step uses).
__device__ __forceinline__ Region region_of(const Dev& P, int slot) {
  if (P.nscenes == 0) {
    Region r;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      r.bmin[a] = P.bmin[a];
      r.bmax[a] = P.bmax[a];
    }
    r.dimx = P.dimx;
    r.dimy = P.dimy;
    r.dimz = P.dimz;
    r.key0 = 0u;
    return r;
  }
  int lo = 0, hi = P.nscenes - 1;  // the last scene whose first slot is <= slot
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(P.scene_first + mid) <= (uint32_t)slot) lo = mid;
    else hi = mid - 1;
  }
  return P.scenes[lo];
}

// ---------------- exact scalar helpers ----------------
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdiv_rn(a, b); }

// Policy-selected ops.
template <bool X> __device__ __forceinline__ float A(float a, float b) { return X ? __fadd_rn(a, b) : a + b; }
template <bool X> __device__ __forceinline__ float S(float a, float b) { return X ? __fsub_rn(a, b) : a - b; }
template <bool X> __device__ __forceinline__ float M(float a, float b) { return X ? __fmul_rn(a, b) : a * b; }
template <bool X> __device__ __forceinline__ float D(float a, float b) { return X ? __fdiv_rn(a, b) : __fdividef(a, b); }
template <bool X> __device__ __forceinline__ float SQ(float a) {
  if (X) return __fsqrt_rn(a);
  return a > 0.0f ? a * rsqrtf(a) : 0.0f;
}

// dot(r, r) from 0 in x, y, z order (vec.h:476-483, 490-494)
template <bool X> __device__ __forceinline__ float mag2(float x, float y, float z) {
  if (X) return __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
  return fmaf(z, z, fmaf(y, y, x * x));
}

// Poly6 3D (kernels.h:64-70): norm*(h^2-r^2)^3, 0 for r > h.
template <bool X> __device__ __forceinline__ float poly6(const Dev& P, float r) {
  if (r > P.h) return 0.0f;
  if (X) {
    const float a = __fsub_rn(__fmul_rn(P.h, P.h), __fmul_rn(r, r));
    return __fmul_rn(__fmul_rn(__fmul_rn(P.poly6_norm, a), a), a);
  }
  const float a = fmaf(-r, r, P.h * P.h);
  return P.poly6_norm * a * a * a;
}

// Scalar factor f of Del_Spikey 3D (kernels.h:163-172) such that the gradient
// is f*r in fast mode; exact mode evaluates component-wise as the reference:
// ((norm*(h-r))*(h-r) * r_i) / (r + FLT_EPSILON).
template <bool X> __device__ __forceinline__ float3 del_spikey(const Dev& P, float rx, float ry,
                                                               float rz, float rm) {
  if (rm > P.h) return make_float3(0.0f, 0.0f, 0.0f);
  if (X) {
    const float hr = __fsub_rn(P.h, rm);
    const float s = __fmul_rn(__fmul_rn(P.spikey_norm, hr), hr);
    const float den = __fadd_rn(rm, FLT_EPSILON);
    return make_float3(__fdiv_rn(__fmul_rn(s, rx), den), __fdiv_rn(__fmul_rn(s, ry), den),
                       __fdiv_rn(__fmul_rn(s, rz), den));
  }
  const float hr = P.h - rm;
  const float f = P.spikey_norm * hr * hr * __fdividef(1.0f, rm + FLT_EPSILON);
  return make_float3(f * rx, f * ry, f * rz);
}

// C_Spline 3D (kernels.h:220-228); the r <= h/2 branch is a double expression.
template <bool X> __device__ __forceinline__ float c_spline(const Dev& P, float r) {
  const float h = P.h;
  if (r > h) return 0.0f;
  if (r <= __fmul_rn(h, 0.5f)) {
    const float hr = __fsub_rn(h, r);
    const double t = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(2.0, (double)hr), (double)hr),
                                                   (double)hr), (double)r), (double)r);
    const double t2 = __dmul_rn(t, (double)r);
    const float h6 = __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(h, h), h), h), h), h), 64.0f);
    return (float)__dmul_rn((double)P.cspline_norm, __dsub_rn(t2, (double)h6));
  }
  const float hr = __fsub_rn(h, r);
  float v = __fmul_rn(P.cspline_norm, hr);
  v = __fmul_rn(v, hr);
  v = __fmul_rn(v, hr);
  v = __fmul_rn(v, r);
  v = __fmul_rn(v, r);
  return __fmul_rn(v, r);
}

// apply_boundary_conditions (particles.h:510-526), always exact; the mover
// sphere is shared, the box is the particle's scene's.
__device__ __forceinline__ float3 boundary(const Dev& P, const Region& R, float3 p) {
  const float dx = xsub(p.x, P.mc[0]), dy = xsub(p.y, P.mc[1]), dz = xsub(p.z, P.mc[2]);
  const float dr2 = mag2<true>(dx, dy, dz);
  if (dr2 < P.mr2) {
    const float dr = __fsqrt_rn(dr2);
    const float a = xsub(P.mr, dr);
    p.x = xadd(p.x, xdiv(xmul(a, dx), dr));
    p.y = xadd(p.y, xdiv(xmul(a, dy), dr));
    p.z = xadd(p.z, xdiv(xmul(a, dz), dr));
  }
  // clamp_in_place (utility_math.h:52-57)
  p.x = p.x < R.bmin[0] ? R.bmin[0] : (p.x > R.bmax[0] ? R.bmax[0] : p.x);
  p.y = p.y < R.bmin[1] ? R.bmin[1] : (p.y > R.bmax[1] ? R.bmax[1] : p.y);
  p.z = p.z < R.bmin[2] ? R.bmin[2] : (p.z > R.bmax[2] ? R.bmax[2] : p.z);
  return p;
}

// floor((c + s)/s) per axis (neighbors.h:109-114).  Returns false when the
// coordinate is non-finite or lands outside the grid; ok grids (checked at
// context creation) never do for clamped positions.
__device__ __forceinline__ int dev_axis_bin(float c, float s) {
  return (int)floorf(xdiv(xadd(c, s), s));
}

// Bin key in the particle's scene's grid (id = Dx*Dy*z + (y*Dx + x),
// neighbors.h:109-114), offset by the scene's first key.
__device__ __forceinline__ bool bin_of(const Dev& P, const Region& R, float x, float y, float z, uint32_t& out) {
  const int bx = dev_axis_bin(x, P.s), by = dev_axis_bin(y, P.s), bz = dev_axis_bin(z, P.s);
  const bool ok = bx >= 0 && by >= 0 && bz >= 0 && bx < R.dimx && by < R.dimy && bz < R.dimz &&
                  isfinite(x) && isfinite(y) && isfinite(z);
  const int cx = min(max(bx, 0), R.dimx - 1), cy = min(max(by, 0), R.dimy - 1),
            cz = min(max(bz, 0), R.dimz - 1);
  out = R.key0 + (uint32_t)(R.dimx * R.dimy) * (uint32_t)cz + ((uint32_t)cy * (uint32_t)R.dimx + (uint32_t)cx);
  return ok;
}

}  // namespace pbf
