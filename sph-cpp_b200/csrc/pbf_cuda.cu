// libpbf_b200: the position-based-fluids step of AdamSimpson/SPH-CPP
// (Simulation/Source/particles.h, neighbors.h; stage order main.cpp:71-124)
// as hand-written sm_100a kernels behind the C ABI of include/pbf.h.
//
// Data layout in HBM (capacity C particles, all 16-byte aligned float4 SoA):
//   home buffers, persistent between steps, in the order of the last cell sort
//     posH  (x, -)     pstH (x*, -)     velH (v, rho)     scrH (scratch Vec, |.|)
//     lamH  float      origH uint32 (reference particle index of each slot)
//   working buffers in the current step's sorted order
//     posS, pstS, velS, origS, velT, xl = (x*, lambda) or (x*, |omega|)
//   grid:   cell_count[B], cell_start[B+1] (begin/end of every bin),
//           key/rank per particle, pairs[C] = (reference index << 32 | slot)
//   lists:  nbr[cap][C] int32 slot indices (column-major: one warp reads one
//           128-byte line per list entry), cnt[C]
//
// One step (pbf_step) is one CUDA graph of:
//   memset counts -> ext+predict+hash+histogram -> 3-pass scan -> scatter ->
//   per-cell stable fix-up -> reorder -> fill lists ->
//   K x [density+lambda, delta-p+x* update (+ velocity on the last)] ->
//   viscosity -> vorticity -> vorticity apply -> viscosity + x = x*.
// Particles are kept in cell order between steps, so neighbours of a warp's
// particles sit in a few contiguous slot ranges (L1/L2 reuse); the reference
// index of every slot (origH) maps results back for downloads and parity.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pbf.h"
#include "pbf_internal.h"
#include "pbf_kernels.cuh"
#include "pbf_fast.cuh"
#include "pbf_learn.cuh"
#include "pbf_mlp_tc.cuh"
#include "pbf_train_tc.cuh"

using pbf::Dev;
using pbf::Fast;

namespace {

constexpr int kBlock = 256;
// density/lambda and delta-p are held to 42 registers (6 blocks of kBlock, or
// 12 of the autotuned 128, per SM): measured faster than at their natural
// 44-48; the other gathers are faster as the compiler leaves them.
constexpr int kGatherMinBlocks = 6;
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

inline int blocks_for(size_t n, int b = kBlock) { return (int)((n + b - 1) / b); }

// Digit histogram entries of the radix sort for up to `capacity` particles
// (2^kRadixBits digits per 2^kRadixTileLog2-element tile); the constants are
// checked against the kernels' below.
constexpr int kRadixBitsHost = 11, kRadixTileHost = 4096;
inline size_t radix_entries(size_t capacity) {
  return ((capacity + kRadixTileHost - 1) / kRadixTileHost) * ((size_t)1 << kRadixBitsHost);
}
// Neighbor list rows are kListAlign-entry multiples long, so the fast gathers
// read whole vectors of indices (the entries past a particle's count are
// replaced by a dummy slot, one past the last particle, whose every kernel
// term is exactly zero).
constexpr int kListAlign = 32;
inline size_t list_stride(int cap) { return ((size_t)cap + kListAlign - 1) / kListAlign * kListAlign; }

// Passes to sort keys < nbins.
inline int radix_passes_for(int nbins) {
  int bits = 0;
  while (bits < 31 && ((int64_t)1 << bits) < (int64_t)nbins) ++bits;
  return (bits + kRadixBitsHost - 1) / kRadixBitsHost;
}

// ============================================================================
// Kernels
// ============================================================================

// Upload: AoS float3 host layout -> float4 home buffers, identity order.
// The dummy slot n the list padding points at: far from every particle (all
// kernel terms vanish: Poly6 and Spiky are 0 beyond h, lambda and |w| are 0),
// unit density (XSPH divides by it).  Kernels only write slots < n.
constexpr float kFar = 1e15f;

__global__ void k_upload(int n, const float* __restrict__ x, const float* __restrict__ v,
                         float4* posH, float4* pstH, float4* velH, float4* scrH, float* lamH,
                         uint32_t* origH, float4* pstS, float4* xl, float4* velS, float4* velT) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    pstS[n] = make_float4(kFar, kFar, kFar, 0.0f);
    xl[n] = make_float4(kFar, kFar, kFar, 0.0f);
    velS[n] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    velT[n] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
  }
  if (i >= n) return;
  const float4 p = make_float4(x[3 * i], x[3 * i + 1], x[3 * i + 2], 0.0f);
  posH[i] = p;
  pstH[i] = p;
  velH[i] = v ? make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.0f) : make_float4(0.f, 0.f, 0.f, 0.f);
  scrH[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  lamH[i] = 0.0f;
  origH[i] = (uint32_t)i;
}

// Particles::add (particles.h:184-199) for k particles at the end: slots and
// reference indices n0 .. n0+k-1, x* = x, v given or zero; the dummy slot
// moves to the new end.
__global__ void k_append(int n0, int k, const float* __restrict__ x, const float* __restrict__ v, float4* posH,
                         float4* pstH, float4* velH, float4* scrH, float* lamH, float* lamsumH, uint32_t* origH,
                         float4* pstS, float4* xl, float4* velS, float4* velT) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = n0 + k;
  if (i == 0) {
    pstS[n] = make_float4(kFar, kFar, kFar, 0.0f);
    xl[n] = make_float4(kFar, kFar, kFar, 0.0f);
    velS[n] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    velT[n] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
  }
  if (i >= k) return;
  const int a = n0 + i;
  const float4 p = make_float4(x[3 * i], x[3 * i + 1], x[3 * i + 2], 0.0f);
  posH[a] = p;
  pstH[a] = p;
  velH[a] = v ? make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.0f) : make_float4(0.f, 0.f, 0.f, 0.f);
  scrH[a] = make_float4(0.f, 0.f, 0.f, 0.f);
  lamH[a] = 0.0f;
  lamsumH[a] = 0.0f;
  origH[a] = (uint32_t)a;
}

// Home slot order -> reference order, AoS float3.
__global__ void k_unpermute_vec(int n, const float4* __restrict__ src, const uint32_t* __restrict__ orig,
                                float* dst) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const float4 v = src[b];
  const uint32_t o = orig[b];
  dst[3 * (size_t)o] = v.x;
  dst[3 * (size_t)o + 1] = v.y;
  dst[3 * (size_t)o + 2] = v.z;
}

// component 3 of a float4 array, or a float array, -> reference order
__global__ void k_unpermute_w(int n, const float4* __restrict__ src4, const float* __restrict__ src1,
                              const uint32_t* __restrict__ orig, float* dst) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  dst[orig[b]] = src4 ? src4[b].w : src1[b];
}

// reference order AoS float3 -> home slot order (w kept)
__global__ void k_permute_vec_in(int n, const float* __restrict__ src, const uint32_t* __restrict__ orig,
                                 float4* dst) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const size_t o = orig[b];
  float4 d = dst[b];
  d.x = src[3 * o];
  d.y = src[3 * o + 1];
  d.z = src[3 * o + 2];
  dst[b] = d;
}

__global__ void k_permute_w_in(int n, const float* __restrict__ src, const uint32_t* __restrict__ orig,
                               float4* dst4, float* dst1) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const float v = src[orig[b]];
  if (dst4) dst4[b].w = v; else dst1[b] = v;
}

// apply_external_forces (particles.h:263-270)
__global__ void k_external(Dev P, int n, float4* vel) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n || !pbf::in_span(P, a)) return;
  vel[a].y = pbf::xadd(vel[a].y, P.gdt);
}

// predict_positions (particles.h:275-287): x* = BC(x + v*dt)
__device__ __forceinline__ float3 predict(const Dev& P, const pbf::Region& R, float4 x, float4 v) {
  float3 s;
  s.x = pbf::xadd(x.x, pbf::xmul(v.x, P.dt));
  s.y = pbf::xadd(x.y, pbf::xmul(v.y, P.dt));
  s.z = pbf::xadd(x.z, pbf::xmul(v.z, P.dt));
  return pbf::boundary(P, R, s);
}

__global__ void k_predict(Dev P, int n, const float4* __restrict__ pos, const float4* __restrict__ vel,
                          float4* pst) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n || !pbf::in_span(P, a)) return;
  const float3 s = predict(P, pbf::region_of(P, a), pos[a], vel[a]);
  pst[a] = make_float4(s.x, s.y, s.z, 0.0f);
}

// Bins holding more particles than this walk their candidates run by run.
constexpr uint32_t kRunBin = 512;

// calculate_bins (neighbors.h:120-125) + bin histogram; the radix sort's
// input (key, pair) goes to the particle's reference index.  The word after
// the histogram (cell_count[nbins]) is raised when a bin passes kRunBin
// particles: only then does the list fill need the runs (k_runs).  The lanes
// of a warp with the same key add to its count once (a settled dam piles
// hundreds of thousands of particles into one bin, whose count would
// otherwise take one atomic per particle, one after another).
__device__ __forceinline__ void hash_out(const Dev& P, int a, uint32_t k, const uint32_t* __restrict__ orig,
                                         uint32_t* key, uint32_t* cell_count, uint32_t* key_ref,
                                         unsigned long long* pair_ref) {
  key[a] = k;
  const unsigned same = __match_any_sync(__activemask(), k);
  if ((threadIdx.x & 31) == (unsigned)(__ffs(same) - 1)) {
    const uint32_t add = (uint32_t)__popc(same), old = atomicAdd(&cell_count[k], add);
    if (old <= kRunBin && old + add > kRunBin) atomicOr(&cell_count[P.nbins], 1u);
  }
  const uint32_t o = orig[a];
  key_ref[o] = k;
  pair_ref[o] = ((unsigned long long)o << 32) | (unsigned long long)(uint32_t)a;
}

__global__ void k_hash(Dev P, int n, const float4* __restrict__ pst, const uint32_t* __restrict__ orig,
                       uint32_t* key, uint32_t* cell_count, uint32_t* key_ref, unsigned long long* pair_ref,
                       uint32_t* err) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const float4 s = pst[a];
  uint32_t k;
  if (!pbf::bin_of(P, pbf::region_of(P, a), s.x, s.y, s.z, k)) atomicOr(err, PBF_FLAG_KEY_RANGE);
  hash_out(P, a, k, orig, key, cell_count, key_ref, pair_ref);
}

// Fused apply_external_forces + predict_positions + calculate_bins + histogram.
__global__ void k_ext_predict_hash(Dev P, int n, const float4* __restrict__ pos, float4* vel, float4* pst,
                                   const uint32_t* __restrict__ orig, uint32_t* key, uint32_t* cell_count,
                                   uint32_t* key_ref, unsigned long long* pair_ref, uint32_t* err) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  float4 v = vel[a];
  v.y = pbf::xadd(v.y, P.gdt);
  vel[a] = v;
  const pbf::Region R = pbf::region_of(P, a);
  const float3 s = predict(P, R, pos[a], v);
  pst[a] = make_float4(s.x, s.y, s.z, 0.0f);
  uint32_t k;
  if (!pbf::bin_of(P, R, s.x, s.y, s.z, k)) atomicOr(err, PBF_FLAG_KEY_RANGE);
  hash_out(P, a, k, orig, key, cell_count, key_ref, pair_ref);
}

// ---- exclusive scan of cell_count[0..m-1] (+ total at [m]) -> cell_start ----
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums,
                                                         uint32_t& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    uint32_t w = lane < nw ? warp_sums[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) warp_sums[lane] = w;
  }
  __syncthreads();
  const uint32_t warp_prefix = wid > 0 ? warp_sums[wid - 1] : 0u;
  total = warp_sums[(blockDim.x >> 5) - 1];
  return warp_prefix + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t* __restrict__ in, int m,
                                                              uint32_t* partial) {
  __shared__ uint32_t ws[32];
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < (size_t)m) s += in[base + i];
  uint32_t total;
  block_exclusive_scan(s, ws, total);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_partials(uint32_t* partial, int np) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < np; base += kScanThreads) {
    const int i = base + threadIdx.x;
    const uint32_t v = i < np ? partial[i] : 0u;
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(v, ws, total);
    const uint32_t c = carry;
    if (i < np) partial[i] = ex + c;
    __syncthreads();
    if (threadIdx.x == 0) carry = c + total;
    __syncthreads();
  }
}

// out[0..m] (m+1 entries): exclusive prefix of in[0..m-1], out[m] = total.
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const uint32_t* __restrict__ in, int m,
                                                             const uint32_t* __restrict__ partial,
                                                             uint32_t* out) {
  __shared__ uint32_t ws[32];
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = base + i < (size_t)m ? in[base + i] : 0u;
    s += v[i];
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan(s, ws, total) + partial[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i <= (size_t)m) out[base + i] = run;
    run += v[i];
  }
}

// ---- stable LSD radix sort of (bin key, pair) ----
// The hash kernels write every particle's key and pair (reference index << 32
// | home slot) at its reference index, so the input is in reference-index
// order and a stable sort by key orders every bin by reference index: the
// permutation of the reference's stable sort_by_key (neighbors.h:130-132).
// kRadixBits-bit digits, least significant first; each pass is a per-tile
// digit histogram (digit-major: hist[d * tiles + tile]), an exclusive scan of
// it (the scan kernels above) and a stable scatter.  The work is O(n) per pass
// however the particles crowd into bins.
constexpr int kRadixBits = 11;
constexpr int kRadixDigits = 1 << kRadixBits;
constexpr int kRadixThreads = 256;
constexpr int kRadixWarps = kRadixThreads / 32;
constexpr int kRadixItems = 16;
constexpr int kRadixTile = kRadixThreads * kRadixItems;  // elements per tile (block)
static_assert(kRadixBits == kRadixBitsHost && kRadixTile == kRadixTileHost, "radix buffer sizing");

__device__ __forceinline__ uint32_t radix_digit(uint32_t key, int shift) {
  return (key >> shift) & (uint32_t)(kRadixDigits - 1);
}

__global__ void __launch_bounds__(kRadixThreads) k_radix_hist(const uint32_t* __restrict__ keys, int n, int shift,
                                                             int tiles, uint32_t* hist) {
  __shared__ uint32_t cnt[kRadixDigits];
  for (int d = threadIdx.x; d < kRadixDigits; d += kRadixThreads) cnt[d] = 0u;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * kRadixTile;
  const int lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kRadixTile; i += kRadixThreads) {  // warp-uniform trip count
    const size_t j = base + i;
    const bool live = j < (size_t)n;
    const uint32_t d = live ? radix_digit(keys[j], shift) : (uint32_t)kRadixDigits;
    const unsigned peers = __match_any_sync(0xffffffffu, d);  // one shared-memory add per distinct digit
    if (live && (peers & ((1u << lane) - 1u)) == 0u) atomicAdd(&cnt[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadixDigits; d += kRadixThreads) hist[(size_t)d * tiles + blockIdx.x] = cnt[d];
}

// Stable scatter of one tile.  Warp w owns elements [w*32*kRadixItems,
// (w+1)*32*kRadixItems) of the tile, walked item by item (element = item*32 +
// lane): equal digits in one item are ranked by lane (__match_any_sync) and a
// per-warp running count per digit carries the rank across items; the warps'
// counts then become exclusive prefixes over the warps, so ranks follow the
// element order across the tile, and tiles follow each other through the
// scanned histogram.  keys_out may be null (last pass).
__global__ void __launch_bounds__(kRadixThreads) k_radix_scatter(const uint32_t* __restrict__ keys_in,
                                                                const unsigned long long* __restrict__ vals_in,
                                                                int n, int shift, int tiles,
                                                                const uint32_t* __restrict__ offsets,
                                                                uint32_t* keys_out, unsigned long long* vals_out) {
  __shared__ uint16_t wcnt[kRadixWarps * kRadixDigits];  // counts <= 32*kRadixItems, prefixes <= kRadixTile
  for (int d = threadIdx.x; d < kRadixWarps * kRadixDigits; d += kRadixThreads) wcnt[d] = 0;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  uint16_t* mine = wcnt + warp * kRadixDigits;
  const size_t wbase = (size_t)blockIdx.x * kRadixTile + (size_t)warp * 32 * kRadixItems;
  uint32_t dig[kRadixItems], rk[kRadixItems];
#pragma unroll
  for (int it = 0; it < kRadixItems; ++it) {
    const size_t j = wbase + (size_t)it * 32 + lane;
    const bool live = j < (size_t)n;
    const uint32_t d = live ? radix_digit(keys_in[j], shift) : (uint32_t)kRadixDigits;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const uint32_t base = live ? (uint32_t)mine[d] : 0u;
    __syncwarp();
    if (live && (peers & lt) == 0u) mine[d] = (uint16_t)(base + (uint32_t)__popc(peers));
    __syncwarp();
    dig[it] = d;
    rk[it] = base + (uint32_t)__popc(peers & lt);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadixDigits; d += kRadixThreads) {
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kRadixWarps; ++w) {
      const uint32_t c = wcnt[w * kRadixDigits + d];
      wcnt[w * kRadixDigits + d] = (uint16_t)run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < kRadixItems; ++it) {
    const size_t j = wbase + (size_t)it * 32 + lane;
    if (j >= (size_t)n) continue;
    const uint32_t d = dig[it];
    const uint32_t pos = offsets[(size_t)d * tiles + blockIdx.x] + (uint32_t)mine[d] + rk[it];
    vals_out[pos] = vals_in[j];
    if (keys_out) keys_out[pos] = keys_in[j];
  }
}

// Gather the state into sorted order.  FULL = also scratch and lambda (the
// per-stage path, where every reference array must follow its particle); the
// fused step passes the learned warm start's lambda sums as lamH/lamS.
template <bool FULL>
__global__ void k_reorder(int n, const unsigned long long* __restrict__ pairs, const uint32_t* __restrict__ key,
                          const float4* __restrict__ posH, const float4* __restrict__ pstH,
                          const float4* __restrict__ velH, const float4* __restrict__ scrH,
                          const float* __restrict__ lamH, float4* posS, float4* pstS, float4* velS,
                          float4* scrS, float* lamS, uint32_t* origS, uint32_t* keyH) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const unsigned long long pr = pairs[b];
  const uint32_t a = (uint32_t)(pr & 0xffffffffull);
  origS[b] = (uint32_t)(pr >> 32);
  keyH[b] = key[a];
  posS[b] = posH[a];
  pstS[b] = pstH[a];
  velS[b] = velH[a];
  if (FULL) scrS[b] = scrH[a];
  if (lamS) lamS[b] = lamH[a];  // FULL: lambda; fused step: last step's lambda sum, when kept
}

// Runs of bit-identical x* among consecutive sorted slots (particles piled
// onto one point, e.g. clamped into a box corner by a collapsing scene):
// run_end[i] = the first slot j > i whose x* differs from slot j - 1's, or the
// end of i's block of kRunBlock slots, whichever comes first.  Equal x* gives
// equal distance tests, so the list fill decides a whole run with one test.
// crowded (may be null): the histogram's flag; zero means no bin is large
// enough for the fill to read the runs, and the launch returns at once.
constexpr int kRunBlock = 1024;
__global__ void __launch_bounds__(kRunBlock) k_runs(int n, const float4* __restrict__ pst, uint32_t* run_end,
                                                    const uint32_t* __restrict__ crowded) {
  if (crowded && *crowded == 0u) return;
  __shared__ uint32_t wfirst[kRunBlock / 32];  // first run start of every warp's 32 slots
  const int i = blockIdx.x * kRunBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t base = (uint32_t)blockIdx.x * kRunBlock;
  const uint32_t bend = min(base + (uint32_t)kRunBlock, (uint32_t)n);
  bool start = false;
  if (i < n) {
    if (threadIdx.x == 0) {
      start = true;
    } else {
      const float4 a = pst[i], b = pst[i - 1];
      start = __float_as_uint(a.x) != __float_as_uint(b.x) || __float_as_uint(a.y) != __float_as_uint(b.y) ||
              __float_as_uint(a.z) != __float_as_uint(b.z);
    }
  }
  const unsigned m = __ballot_sync(0xffffffffu, start);
  if (lane == 0) wfirst[w] = m ? base + (uint32_t)(w * 32 + __ffs(m) - 1) : 0xffffffffu;
  __syncthreads();
  if (i >= n) return;
  const unsigned above = m & ~((2u << lane) - 1u);  // starts in this warp after slot i
  uint32_t e = bend;
  if (above) {
    e = base + (uint32_t)(w * 32 + __ffs(above) - 1);
  } else {
    for (int v = w + 1; v < kRunBlock / 32; ++v)
      if (wfirst[v] != 0xffffffffu) {
        e = wfirst[v];
        break;
      }
  }
  run_end[i] = e;
}


// One crowded bin [q0, q1) of the list fill, run by run: one distance test per
// run of bit-identical x*; on a hit the run's slots are appended in order, the
// particle's own slot left out, while the list has room.  Returns the new
// length.  Out of line, so that the common per-candidate loop keeps its code.
__device__ __noinline__ int fill_runs(float px, float py, float pz, float s2, int cap, uint32_t self, uint32_t q0,
                                      uint32_t q1, const float4* __restrict__ pst,
                                      const uint32_t* __restrict__ run_end, int32_t* row, uint16_t* row16, int off,
                                      int count) {
  for (uint32_t q = q0; q < q1;) {
    const float4 xq = pst[q];
    const uint32_t qe = min(run_end[q], q1);
    const float d2 = pbf::mag2<true>(pbf::xsub(px, xq.x), pbf::xsub(py, xq.y), pbf::xsub(pz, xq.z));
    if (d2 < s2) {
      for (uint32_t r = q; r < qe && count < cap; ++r) {
        if (r == self) continue;
        if (row16) row16[count] = (uint16_t)((int)r + off);
        row[pbf::list_off(count++)] = (int32_t)r;
      }
      if (count >= cap) break;
    }
    q = qe;
  }
  return count;
}

// fill_neighbors (neighbors.h:197-230) over slots in sorted order: the 27
// bins in the reference's order (x offset outer, z inner, float re-hash of
// coord + i*s), candidates of a bin in ascending reference index, strict
// d^2 < s^2, self skipped, the first `cap` kept.  Each thread fills its own
// list in the warp-tiled layout (pbf::list_off).  A neighbour bin whose every point is provably
// farther than s from the particle is skipped: the per-axis distance from the
// particle to the bin's face, less a margin of many ulps of the coordinate
// (P.skip_eps), squared and summed, exceeds s^2.  Only bins equal to the
// integer offset of the particle's own bin are skipped, so the reference's
// float re-hash still decides which bins are visited.  A bin of more than
// kRunBin particles is walked run by run (k_runs): a run of bit-identical x*
// is one distance test, and on a hit its slots are appended in order (the
// particle's own slot left out), the list the one-by-one walk gives.
constexpr int kFillBlock = 128;

// Tiles of kTile consecutive sorted slots (one warp of the list fill, one
// block of the staged gathers).  A tile's neighbour bins lie in the bounding
// box of its own bins grown by one bin; every (y, z) row of that box is one
// contiguous slot run (bins of a row have consecutive keys), so a staged
// gather copies at most kTileRuns runs, kStageMax records, to shared memory.
constexpr int kTile = 32, kTileRuns = 16, kStageMax = 1024;

// Staging descriptors of the tiles (written by the list fill).
struct TileIO {
  int32_t* nruns;   // [tiles] runs of the tile; 0: not staged (the gathers walk the int32 lists)
  int32_t* total;   // [tiles] staged records
  int4* runs;       // [tiles][kTileRuns] (first slot, records, staging base, 0)
  uint16_t* nbr16;  // [slot][stride] staging index of every list entry
};

// The tile's staging box (STAGE): the runs of the own bins grown by one bin.
struct FillStage {
  bool staged;
  int xmn, xmx, ymn, zmn, ny, nz;
  uint16_t* row16;
};

// One visit of the list fill: bin (cx, cy, cz) of the particle's scene, its
// candidates in ascending slot order, strict d^2 < s^2, self skipped, while
// the list has room.  A bin at the integer offset of the particle's own bin
// (at_offset) whose every point is provably farther than s (e2, the squared
// distance to its faces less the margin, above s^2) is skipped; a crowded
// bin goes run by run.  Returns the list's new length.
template <bool STAGE>
__device__ __forceinline__ int fill_visit(int cx, int cy, int cz, bool at_offset, float e2, float px, float py,
                                          float pz, bool finite, const pbf::Region& R, float s2, int cap,
                                          uint32_t self, const uint32_t* __restrict__ cell_start,
                                          const float4* __restrict__ pst, const uint32_t* __restrict__ run_end,
                                          int32_t* row, uint32_t* err, const FillStage& S, const int* soff,
                                          bool& stray, int count) {
  if (!finite || cx < 0 || cy < 0 || cz < 0 || cx >= R.dimx || cy >= R.dimy || cz >= R.dimz) {
    atomicOr(err, PBF_FLAG_KEY_RANGE);
    return count;
  }
  if (at_offset && e2 > s2) return count;
  const uint32_t nb =
      R.key0 + (uint32_t)(R.dimx * R.dimy) * (uint32_t)cz + ((uint32_t)cy * (uint32_t)R.dimx + (uint32_t)cx);
  const bool staged = STAGE && S.staged;
  int off = 0;
  if (staged) {
    const int ry = cy - (S.ymn - 1), rz = cz - (S.zmn - 1);
    if (cx < S.xmn - 1 || cx > S.xmx + 1 || ry < 0 || ry >= S.ny || rz < 0 || rz >= S.nz) stray = true;
    else off = soff[(threadIdx.x & ~31) + rz * S.ny + ry];
  }
  const uint32_t q0 = cell_start[nb], q1 = cell_start[nb + 1];
  if (q1 - q0 > kRunBin) {
    count = fill_runs(px, py, pz, s2, cap, self, q0, q1, pst, run_end, row, staged ? S.row16 : nullptr, off, count);
  } else if (q0 <= self && self < q1) {  // the particle's own bin: skip itself
    for (uint32_t q = q0; q < q1; ++q) {
      const float4 xq = pst[q];
      const float d2 = pbf::mag2<true>(pbf::xsub(px, xq.x), pbf::xsub(py, xq.y), pbf::xsub(pz, xq.z));
      if (d2 < s2 && q != self && count < cap) {
        if (staged) S.row16[count] = (uint16_t)((int)q + off);
        row[pbf::list_off(count++)] = (int32_t)q;
      }
    }
  } else {  // another bin (all but one of the 27, at the same offset for every lane)
    for (uint32_t q = q0; q < q1; ++q) {
      const float4 xq = pst[q];
      const float d2 = pbf::mag2<true>(pbf::xsub(px, xq.x), pbf::xsub(py, xq.y), pbf::xsub(pz, xq.z));
      if (d2 < s2 && count < cap) {
        if (staged) S.row16[count] = (uint16_t)((int)q + off);
        row[pbf::list_off(count++)] = (int32_t)q;
      }
    }
  }
  return count;
}

// calculate_neighbor_indices (neighbors.h:172-185): the bin of coord + i*s
// along one axis for i = -1, 0, 1, in the reference's float operations.  The
// 27 bins combine these per-axis values, so 9 float hashes cover all of them.
__device__ __forceinline__ void axis_bins(float c, float s, int (&out)[3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) out[i] = pbf::dev_axis_bin(pbf::xadd(c, pbf::xmul((float)(i - 1), s)), s);
}

// The 27 visits of one particle, in the reference's order (x offset outer,
// z inner) or, slot, z offset outer and x inner: the bins then come in
// ascending keys, so a warp's lanes read neighbouring slots together in the
// gathers.  slot records where each visit's entries start (sc[visit
// k*9 + j*3 + i]).  Stops at the cap and returns the list's length.  The
// order is a run-time choice in one loop: two compiled walks made the fill
// of a settled dam (crowded bins) 10-25% slower.
template <bool STAGE>
__device__ __forceinline__ int fill_walk(float px, float py, float pz, const int (&bx)[3], const int (&by)[3],
                                         const int (&bz)[3], float s, float skip_eps, const pbf::Region& R,
                                         float s2, int cap, uint32_t self, const uint32_t* __restrict__ cell_start,
                                         const float4* __restrict__ pst, const uint32_t* __restrict__ run_end,
                                         int32_t* row, uint32_t* err, const FillStage& S, const int* soff,
                                         bool& stray, bool slot, uint8_t* sc) {
  const bool finite = isfinite(px) && isfinite(py) && isfinite(pz);
  // per-axis distance from the particle to its own bin's faces, less the margin
  const float lo[3] = {fmaxf(px - ((float)bx[1] * s - s) - skip_eps, 0.f),
                       fmaxf(py - ((float)by[1] * s - s) - skip_eps, 0.f),
                       fmaxf(pz - ((float)bz[1] * s - s) - skip_eps, 0.f)};
  const float hi[3] = {fmaxf(((float)(bx[1] + 1) * s - s) - px - skip_eps, 0.f),
                       fmaxf(((float)(by[1] + 1) * s - s) - py - skip_eps, 0.f),
                       fmaxf(((float)(bz[1] + 1) * s - s) - pz - skip_eps, 0.f)};
  int count = 0;
  for (int u = 0; u < 3; u++) {
    for (int j = 0; j < 3; j++) {
      for (int w = 0; w < 3; w++) {
        const int i = slot ? w : u, k = slot ? u : w;
        if (slot) sc[k * 9 + j * 3 + i] = (uint8_t)count;
        const float ex = i == 0 ? lo[0] : (i == 2 ? hi[0] : 0.f);
        const float ey = j == 0 ? lo[1] : (j == 2 ? hi[1] : 0.f);
        const float ez = k == 0 ? lo[2] : (k == 2 ? hi[2] : 0.f);
        const int cx = bx[i], cy = by[j], cz = bz[k];
        count = fill_visit<STAGE>(cx, cy, cz, cx == bx[1] + i - 1 && cy == by[1] + j - 1 && cz == bz[1] + k - 1,
                                  ex * ex + ey * ey + ez * ez, px, py, pz, finite, R, s2, cap, self, cell_start, pst,
                                  run_end, row, err, S, soff, stray, count);
        if (count >= cap) return count;
      }
    }
  }
  return count;
}

// Beside each list of the fast path (seg, kSegWords words per slot): where
// each of the 27 visits' entries start, in visit order (z offset outer), then
// kSegReferenceOrder when the list is in the reference's order (the cap is at
// most 64, so a byte holds an offset).
constexpr int kSegWords = 8;
constexpr uint8_t kSegReferenceOrder = 0xFF;

// The fast path's choice of list order, in device words (FillWord): the
// lists that reached the cap in the fill under way, the slot-order lists
// queued for the reference's walk, the order of the next fill (1 = slot
// order), the redo kernel's block ticket, and the order the last fill used.
// The cap keeps the first entries in the reference's order, so a slot-order
// list that reaches it is walked again in that order (k_fill_redo).  Once
// more than 1 / kSlotCappedShare of the lists reach the cap (a dam that has
// settled), the fill walks in the reference's order, where the cap costs
// nothing, until the share drops again.  At 1 in 16 or 1 in 8 the re-walks
// cost more than the slot order saves in the gathers.
enum FillWord {
  kFillCapped = 0,
  kFillQueued = 1,
  kFillSlotOrder = 2,
  kFillTicket = 3,
  kFillLastOrder = 4,
  kFillWords = 5
};
constexpr uint32_t kSlotCappedShare = 64;

// The list of slot b (a thread's share of k_fill2).  SLOT (fast math): in
// the order fw chose, the visits' starts or the reference-order mark in seg,
// a slot-order list that reached the cap queued for k_fill_redo; else in the
// reference's order.
template <bool STAGE, bool SLOT>
__device__ __forceinline__ void fill_thread(int b, const Dev& P, int n, size_t stride, const float4* __restrict__ pst,
                                            const uint32_t* __restrict__ cell_start,
                                            const uint32_t* __restrict__ run_end, int32_t* nbr, int32_t* cnt,
                                            uint32_t* err, const TileIO& T, uint32_t* seg, uint32_t* fw,
                                            int32_t* queue) {
  __shared__ __align__(16) uint8_t seg_smem[SLOT ? kFillBlock : 1][4 * kSegWords];
  if (!STAGE && b >= n) return;
  if (STAGE && (b & ~(kTile - 1)) >= n) return;  // a whole warp past the end: no tile (warp-uniform)
  const bool live = b < n;
  const int bb = live ? b : n - 1;  // the lanes past the end of the last tile mirror the last particle
  const float4 xp = pst[bb];
  const int cap = P.cap;
  const float s = P.s;
  const pbf::Region R = pbf::region_of(P, bb);
  int32_t* row = nbr + pbf::list_base(b, stride);
  int bx[3], by[3], bz[3];
  axis_bins(xp.x, s, bx);
  axis_bins(xp.y, s, by);
  axis_bins(xp.z, s, bz);
  const bool finite = isfinite(xp.x) && isfinite(xp.y) && isfinite(xp.z);
  // The tile's staging runs (STAGE): warp-wide box of the own bins, one run
  // per (y, z) row of the grown box, the runs' staging bases by a prefix sum.
  __shared__ int soff[STAGE ? kFillBlock : 1];  // per lane: staging base - first slot of run `lane`
  const int lane = threadIdx.x & 31, tile = b / kTile;
  int xmn = 0, xmx = 0, ymn = 0, zmn = 0, ny = 0, nz = 0;
  bool staged = false, stray = false;
  uint16_t* row16 = STAGE ? T.nbr16 + (size_t)b * stride : nullptr;
  if (STAGE) {
    const unsigned full = 0xffffffffu;
    const uint32_t key0 = __shfl_sync(full, R.key0, 0);  // every lane shuffles
    const bool same = __all_sync(full, finite && R.key0 == key0);
    xmn = __reduce_min_sync(full, (unsigned)bx[1] ^ 0x80000000u) ^ 0x80000000u;
    xmx = __reduce_max_sync(full, (unsigned)bx[1] ^ 0x80000000u) ^ 0x80000000u;
    ymn = __reduce_min_sync(full, (unsigned)by[1] ^ 0x80000000u) ^ 0x80000000u;
    const int ymx = __reduce_max_sync(full, (unsigned)by[1] ^ 0x80000000u) ^ 0x80000000u;
    zmn = __reduce_min_sync(full, (unsigned)bz[1] ^ 0x80000000u) ^ 0x80000000u;
    const int zmx = __reduce_max_sync(full, (unsigned)bz[1] ^ 0x80000000u) ^ 0x80000000u;
    ny = ymx - ymn + 3;
    nz = zmx - zmn + 3;
    staged = same && ny * nz <= kTileRuns;
    int slot0 = 0, len = 0;
    if (staged && lane < ny * nz) {
      const int yr = ymn - 1 + lane % ny, zr = zmn - 1 + lane / ny;
      const int x0 = max(xmn - 1, 0), x1 = min(xmx + 1, R.dimx - 1);
      if (yr >= 0 && yr < R.dimy && zr >= 0 && zr < R.dimz && x0 <= x1) {
        const uint32_t rk = R.key0 + (uint32_t)(R.dimx * R.dimy) * (uint32_t)zr + (uint32_t)yr * (uint32_t)R.dimx;
        slot0 = (int)cell_start[rk + (uint32_t)x0];
        len = (int)cell_start[rk + (uint32_t)x1 + 1u] - slot0;
      }
    }
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(full, incl, o);
      if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(full, incl, 31);
    const int base = incl - len;
    staged = staged && total <= kStageMax;
    soff[threadIdx.x] = base - slot0;
    if (lane == 0) {
      T.nruns[tile] = staged ? ny * nz : 0;
      T.total[tile] = total;
    }
    if (staged && lane < ny * nz) T.runs[(size_t)tile * kTileRuns + lane] = make_int4(slot0, len, base, 0);
    __syncwarp();
    if (!live) return;
  }
  const FillStage S{staged, xmn, xmx, ymn, zmn, ny, nz, row16};
  const bool slot = SLOT && fw[kFillSlotOrder] != 0;
  uint8_t* sc = SLOT ? seg_smem[threadIdx.x] : nullptr;
  const int count = fill_walk<STAGE>(xp.x, xp.y, xp.z, bx, by, bz, s, P.skip_eps, R, P.s2, cap, (uint32_t)b,
                                     cell_start, pst, run_end, row, err, S, soff, stray, slot, sc);
  cnt[b] = count;
  if (SLOT) {
    const bool capped = count >= cap;
    // warp-aggregated counts: the lists at the cap, the slot-order ones among them queued
    const unsigned act = __activemask(), lane_lt = (1u << (threadIdx.x & 31)) - 1u;
    const int leader = __ffs(act) - 1;
    const unsigned cm = __ballot_sync(act, capped), qm = __ballot_sync(act, slot && capped);
    uint32_t qbase = 0;
    if ((int)(threadIdx.x & 31) == leader) {
      if (cm) atomicAdd(&fw[kFillCapped], (uint32_t)__popc(cm));
      if (qm) qbase = atomicAdd(&fw[kFillQueued], (uint32_t)__popc(qm));
    }
    qbase = __shfl_sync(act, qbase, leader);
    if (slot && capped) {
      queue[qbase + __popc(qm & lane_lt)] = b;
      if (STAGE) stray = true;  // the tile walks the int32 lists
    }
    if (slot) {  // (a fill in the reference's order leaves seg alone: the export reads its order word)
      sc[27] = capped ? kSegReferenceOrder : 0;
      const uint32_t* w = reinterpret_cast<const uint32_t*>(seg_smem[threadIdx.x]);
#pragma unroll
      for (int v = 0; v < kSegWords; ++v) seg[(size_t)b * kSegWords + v] = w[v];
    }
  }
  // a bin outside the tile's box (float re-hash at a bin face): the tile walks the int32 lists
  if (STAGE && stray) T.nruns[tile] = 0;
}

template <bool STAGE, bool SLOT>
__global__ void __launch_bounds__(kFillBlock) k_fill2(Dev P, int n, size_t stride, const float4* __restrict__ pst,
                                                      const uint32_t* __restrict__ cell_start,
                                                      const uint32_t* __restrict__ run_end, int32_t* nbr,
                                                      int32_t* cnt, uint32_t* err, TileIO T, uint32_t* seg,
                                                      uint32_t* fw, int32_t* queue) {
  fill_thread<STAGE, SLOT>(blockIdx.x * kFillBlock + threadIdx.x, P, n, stride, pst, cell_start, run_end, nbr, cnt,
                           err, T, seg, fw, queue);
}

// The queued slot-order lists that reached the cap, walked again in the
// reference's order (int32 lists; their seg already says so).  Then the last
// block to finish picks the next fill's order from the share of lists at the
// cap and clears the counts.  No thread returns early: every block reaches
// the ticket.
__global__ void __launch_bounds__(kFillBlock) k_fill_redo(Dev P, int n, size_t stride, const float4* __restrict__ pst,
                                                          const uint32_t* __restrict__ cell_start,
                                                          const uint32_t* __restrict__ run_end, int32_t* nbr,
                                                          int32_t* cnt, uint32_t* err, const int32_t* __restrict__ queue,
                                                          uint32_t* fw) {
  const uint32_t queued = fw[kFillQueued];
  for (uint32_t t = blockIdx.x * kFillBlock + threadIdx.x; t < queued; t += gridDim.x * kFillBlock) {
    const int b = queue[t];
    const float4 xp = pst[b];
    const pbf::Region R = pbf::region_of(P, b);
    int bx[3], by[3], bz[3];
    axis_bins(xp.x, P.s, bx);
    axis_bins(xp.y, P.s, by);
    axis_bins(xp.z, P.s, bz);
    const FillStage none{};
    bool stray = false;
    cnt[b] = fill_walk<false>(xp.x, xp.y, xp.z, bx, by, bz, P.s, P.skip_eps, R, P.s2, P.cap, (uint32_t)b,
                              cell_start, pst, run_end, nbr + pbf::list_base(b, stride), err, none, nullptr,
                              stray, false, nullptr);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&fw[kFillTicket], 1u) == gridDim.x - 1) {
      __threadfence();
      const uint32_t capped = atomicAdd(&fw[kFillCapped], 0u);
      fw[kFillLastOrder] = fw[kFillSlotOrder];
      fw[kFillSlotOrder] = (uint64_t)capped * kSlotCappedShare <= (uint64_t)n ? 1u : 0u;
      fw[kFillCapped] = 0;
      fw[kFillQueued] = 0;
      fw[kFillTicket] = 0;
    }
  }
}

// ---- density (particles.h:292-313) ----
// Per-stage form: writes rho into vel.w.  A particle sitting on a neighbour is
// nudged (particles.h:303-305); the reference writes position_stars_[p] in
// place while other threads read it.  Here each particle sums with its own
// nudged position and every position goes to pst_out, copied back after the
// pass (deterministic: neighbours see nudges from the next stage on).
template <bool X>
__global__ void __launch_bounds__(kBlock) k_density(Dev P, int n, size_t stride, const int32_t* __restrict__ nbr,
                                                    const int32_t* __restrict__ cnt, const float4* __restrict__ pst,
                                                    float4* vel, float4* pst_out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  float4 xp = pst[b];
  if (!pbf::in_span(P, b)) {  // outside the span: x* and rho stay
    pst_out[b] = xp;
    return;
  }
  const int c = cnt[b];
  float rho = pbf::M<X>(P.m, P.W0);
  bool nudged = false;
  for (int k = 0; k < c; ++k) {
    const int q = nbr[pbf::list_at(b, stride, k)];
    const float4 xq = pst[q];
    float rx = pbf::S<X>(xp.x, xq.x), ry = pbf::S<X>(xp.y, xq.y), rz = pbf::S<X>(xp.z, xq.z);
    float rm = pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz));
    if ((double)rm < 0.00000001) {
      const float4 v = vel[b];
      xp.x = pbf::xsub(xp.x, pbf::xdiv(pbf::xmul(v.x, P.dt), 50.0f));
      xp.y = pbf::xsub(xp.y, pbf::xdiv(pbf::xmul(v.y, P.dt), 50.0f));
      xp.z = pbf::xsub(xp.z, pbf::xdiv(pbf::xmul(v.z, P.dt), 50.0f));
      nudged = true;
      rx = pbf::S<X>(xp.x, xq.x); ry = pbf::S<X>(xp.y, xq.y); rz = pbf::S<X>(xp.z, xq.z);
      rm = pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz));
    }
    rho = pbf::A<X>(rho, pbf::M<X>(P.m, pbf::poly6<X>(P, rm)));
  }
  vel[b].w = rho;
  pst_out[b] = xp;
  (void)nudged;
}

// compute_pressure_lambdas (particles.h:318-342), per-stage form.
template <bool X>
__device__ __forceinline__ void lambda_terms(const Dev& P, float rx, float ry, float rz, float rm, float3& sg,
                                             float& sumC) {
  const float3 dw = pbf::del_spikey<X>(P, rx, ry, rz, rm);
  const float gx = pbf::M<X>(P.neg_inv_rho0, dw.x), gy = pbf::M<X>(P.neg_inv_rho0, dw.y),
              gz = pbf::M<X>(P.neg_inv_rho0, dw.z);
  sg.x = pbf::S<X>(sg.x, gx);
  sg.y = pbf::S<X>(sg.y, gy);
  sg.z = pbf::S<X>(sg.z, gz);
  sumC = pbf::A<X>(sumC, pbf::mag2<X>(gx, gy, gz));
}

template <bool X>
__device__ __forceinline__ float lambda_of(const Dev& P, float rho, float3 sg, float sumC) {
  const float constraint = pbf::S<X>(pbf::D<X>(rho, P.rho0), 1.0f);
  const float Cp = constraint < 0.0f ? 0.0f : constraint;
  sumC = pbf::A<X>(sumC, pbf::mag2<X>(sg.x, sg.y, sg.z));
  return pbf::D<X>(-Cp, pbf::A<X>(sumC, P.lambda_eps));
}

template <bool X>
__global__ void __launch_bounds__(kBlock) k_lambda(Dev P, int n, size_t stride, const int32_t* __restrict__ nbr,
                                                   const int32_t* __restrict__ cnt, const float4* __restrict__ pst,
                                                   const float4* __restrict__ vel, float* lam) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n || !pbf::in_span(P, b)) return;
  const float4 xp = pst[b];
  const int c = cnt[b];
  float3 sg = make_float3(0.f, 0.f, 0.f);
  float sumC = 0.0f;
  for (int k = 0; k < c; ++k) {
    const float4 xq = pst[nbr[pbf::list_at(b, stride, k)]];
    const float rx = pbf::S<X>(xp.x, xq.x), ry = pbf::S<X>(xp.y, xq.y), rz = pbf::S<X>(xp.z, xq.z);
    lambda_terms<X>(P, rx, ry, rz, pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz)), sg, sumC);
  }
  lam[b] = lambda_of<X>(P, vel[b].w, sg, sumC);
}

// Fused density + lambda: one neighbour pass computes rho_p and the gradient
// sums (lambda needs only its own density).  Writes xl = (x*, lambda) for the
// delta-p gather, rho into vel.w and lambda into the home lambda array.  When
// a particle sits on a neighbour it is nudged (particles.h:303-305) and the
// launch raises *nudge: k_lambda_fixup then recomputes every lambda from the
// nudged positions, which is what a separate lambda stage after the density
// stage sees.
template <bool X>
__device__ __forceinline__ void density_lambda_one(const Dev& P, int b, size_t stride, const int32_t* __restrict__ nbr,
                                                   const int32_t* __restrict__ cnt, const float4* __restrict__ pst,
                                                   float4* xl, float4* vel, float* lam, uint32_t* nudge) {
  float4 xp = pst[b];
  const int c = cnt[b];
  float rho = pbf::M<X>(P.m, P.W0);
  float3 sg = make_float3(0.f, 0.f, 0.f);
  float sumC = 0.0f;
  bool nudged = false;
  for (int k = 0; k < c; ++k) {
    const float4 xq = pst[nbr[pbf::list_at(b, stride, k)]];
    float rx = pbf::S<X>(xp.x, xq.x), ry = pbf::S<X>(xp.y, xq.y), rz = pbf::S<X>(xp.z, xq.z);
    float rm = pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz));
    if ((double)rm < 0.00000001) {
      const float4 v = vel[b];
      xp.x = pbf::xsub(xp.x, pbf::xdiv(pbf::xmul(v.x, P.dt), 50.0f));
      xp.y = pbf::xsub(xp.y, pbf::xdiv(pbf::xmul(v.y, P.dt), 50.0f));
      xp.z = pbf::xsub(xp.z, pbf::xdiv(pbf::xmul(v.z, P.dt), 50.0f));
      nudged = true;
      rx = pbf::S<X>(xp.x, xq.x); ry = pbf::S<X>(xp.y, xq.y); rz = pbf::S<X>(xp.z, xq.z);
      rm = pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz));
    }
    rho = pbf::A<X>(rho, pbf::M<X>(P.m, pbf::poly6<X>(P, rm)));
    lambda_terms<X>(P, rx, ry, rz, rm, sg, sumC);
  }
  if (nudged) *nudge = 1u;
  const float l = lambda_of<X>(P, rho, sg, sumC);
  xl[b] = make_float4(xp.x, xp.y, xp.z, l);
  vel[b].w = rho;
  lam[b] = l;
}

template <bool X>
__global__ void __launch_bounds__(kBlock) k_density_lambda(Dev P, int n, size_t stride,
                                                           const int32_t* __restrict__ nbr,
                                                           const int32_t* __restrict__ cnt,
                                                           const float4* __restrict__ pst, float4* xl,
                                                           float4* vel, float* lam, uint32_t* nudge) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  density_lambda_one<X>(P, b, stride, nbr, cnt, pst, xl, vel, lam, nudge);
}

// Fast density + lambda (see pbf_fast.cuh), kGL lanes per particle.  A
// particle nudged off a neighbour (particles.h:303-305) is seen at its nudged
// position by the others from the delta-p pass on — the order in which the
// reference's parallel builds see it when every neighbour reads before the
// write; the exact path instead recomputes lambda (k_lambda_fixup).
// Modes: kDlPlain; kDlRecord also writes the learned warm start's features
// (first iteration) and sums the applied lambdas into the label; kDlCheck is
// the learned solver's residual check: skipped once the step has converged,
// else each block writes the sum of its particles' clamped density errors
// to io.partials[blockIdx.x].
enum { kDlPlain = 0, kDlRecord = 1, kDlCheck = 2 };

struct LearnIO {
  float* feats;           // [N][12] raw features (kDlRecord, first iteration)
  float* lamsum;          // lambda applied this step (label / next step's feature)
  const float* lamprev;   // lambda applied last step, in this step's order
  pbf::SolveState* state; // kDlCheck
  double* partials;       // kDlCheck: one sum per block of the (persistent) grid
  int first;              // first Jacobi iteration of the step
  float tol;              // kDlCheck: residual tolerance
  int final_check;        // kDlCheck: the step's last allowed check (records, never extends)
  pbf::SolveLoop loop;    // kDlCheck inside the graph's conditional loop
};

// The sums a density + lambda gather produces for one particle, combined
// over its lane group: sw = sum (h^2 - d^2)^3, s1 = sum (h-r)^2/r * r_vec,
// s2 = sum ((h-r)^2/r)^2 d^2 (the constant factors of grad C are applied once,
// after the walk), the smallest d^2 and (NH) the count of neighbours inside h.
struct DensitySums {
  float sw, s1x, s1y, s1z, s2, dmin, nh;
};

// STAGED: the neighbour records come from the tile's staging area `src` in
// shared memory through the 16-bit list row16; else from `src` in global
// memory through the int32 list row.  `dummy` names the zero record.
template <int GL, bool NH, bool STAGED = false, bool COH = false>
__device__ __forceinline__ DensitySums density_sums(const Fast& F, const pbf::Group& G, const int32_t* row,
                                                    const uint16_t* row16, int c, int dummy, const float4* src,
                                                    float4 xp) {
  DensitySums S{0.f, 0.f, 0.f, 0.f, 0.f, FLT_MAX, 0.f};
  auto body = [&](int, float4 xq) {
    const float dx = xp.x - xq.x, dy = xp.y - xq.y, dz = xp.z - xq.z;
    const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    S.dmin = fminf(S.dmin, d2);
    if (NH) S.nh += d2 < F.h2 ? 1.f : 0.f;
    const float a = fmaxf(F.h2 - d2, 0.0f);
    S.sw = fmaf(a * a, a, S.sw);
    const float t = pbf::spikey_over_r(F, d2);
    S.s1x = fmaf(t, dx, S.s1x);
    S.s1y = fmaf(t, dy, S.s1y);
    S.s1z = fmaf(t, dz, S.s1z);
    S.s2 = fmaf(t * t, d2, S.s2);
  };
  if (STAGED)
    pbf::swalk1<GL>(row16, c, dummy, G.lane, src, body);
  else
    pbf::gwalk1<GL, false, COH>(row, c, dummy, G.lane, src, body);
  S.sw = pbf::gsum<GL>(S.sw);
  S.s1x = pbf::gsum<GL>(S.s1x);
  S.s1y = pbf::gsum<GL>(S.s1y);
  S.s1z = pbf::gsum<GL>(S.s1z);
  S.s2 = pbf::gsum<GL>(S.s2);
  if (NH) S.nh = pbf::gsum<GL>(S.nh);
  S.dmin = pbf::gmin<GL>(S.dmin);
  return S;
}

// COH: inside the persistent step (pbf::ldw).
template <int MODE, int GL, bool STAGED = false, bool COH = false>
__device__ __forceinline__ void density_lambda_tile(int tile, const Dev& P, const Fast& F, int n, size_t stride,
                                                    const int32_t* __restrict__ nbr, const int32_t* __restrict__ cnt,
                                                    const float4* __restrict__ pst, float4* xl, float4* vel,
                                                    float* lam, uint32_t* nudge, const LearnIO& io, float& err,
                                                    const uint16_t* nbr16 = nullptr, const float4* stage = nullptr,
                                                    int staged = 0) {
  const pbf::Group G = pbf::group_at<GL>(n, tile);
  const int b = G.b;
  const float4 xp = pst[b];
  const int c = G.live ? cnt[b] : 0;
  const DensitySums S = density_sums<GL, MODE == kDlRecord, STAGED, COH>(
      F, G, nbr + pbf::list_base(b, stride), STAGED ? nbr16 + (size_t)b * stride : nullptr, c, STAGED ? staged : n,
      STAGED ? stage : pst, xp);
  const float rho = fmaf(F.m_poly, S.sw, F.m_w0);
  if (MODE == kDlCheck && G.live && G.lane == 0) err += fmaxf(fmaf(rho, F.inv_rho0, -1.0f), 0.0f);
  if (!G.live || G.lane != 0) return;
  const float L2 = F.lam_grad * F.lam_grad;
  const float sc = L2 * S.s2;  // sum |grad_q C|^2
  const float g2 = L2 * fmaf(S.s1z, S.s1z, fmaf(S.s1y, S.s1y, S.s1x * S.s1x));  // |grad_p C|^2
  const bool close = S.dmin < 4e-16f;
  const float nh = S.nh;
  if (close) {  // a neighbour (almost) on top: the reference-ordered path decides the nudge
    density_lambda_one<false>(P, b, stride, nbr, cnt, pst, xl, vel, lam, nudge);
  } else {
    const float C = fmaxf(fmaf(rho, F.inv_rho0, -1.0f), 0.0f);
    const float l = -C / (sc + g2 + F.lambda_eps);
    xl[b] = make_float4(xp.x, xp.y, xp.z, l);
    vel[b].w = rho;
    lam[b] = l;
  }
  if (MODE == kDlRecord) {
    if (io.first) {
      float f[pbf::kMlpIn];
      pbf::raw_features(P, pbf::region_of(P, b), F, f, c, rho, sc, g2, (int)nh, io.lamprev[b], vel[b], xp);
#pragma unroll
      for (int k = 0; k < pbf::kMlpIn; ++k) io.feats[(size_t)b * pbf::kMlpIn + k] = f[k];
      io.lamsum[b] = lam[b];
    } else {
      io.lamsum[b] += lam[b];
    }
  }
}

// The residual check runs on a persistent grid walking the tiles, so that
// once the step has converged the launch costs a few hundred empty blocks.
// LOOP: a check inside the graph's conditional loop (pbf::decide_if_last).
// COND: a plain pass of the learned solver's sampled checks, skipped once the
// step has converged.
template <int MODE, int GL, bool LOOP = false, bool COND = false>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) kf_density_lambda(Dev P, Fast F, int n, size_t stride,
                                                            const int32_t* __restrict__ nbr,
                                                            const int32_t* __restrict__ cnt,
                                                            const float4* __restrict__ pst, float4* xl, float4* vel,
                                                            float* lam, uint32_t* nudge, LearnIO io) {
  if (COND && io.state->done) return;
  if (MODE == kDlCheck && io.state->done) {
    // a check after the step converged: it ends the loop it runs in
    if constexpr (LOOP)
      if (io.loop.use && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(io.loop.cond, 0u);
    return;
  }
  const int tiles = pbf::tiles_of<GL>(n);
  float err = 0.0f;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x)
    density_lambda_tile<MODE, GL>(tile, P, F, n, stride, nbr, cnt, pst, xl, vel, lam, nudge, io, err);
  if (MODE == kDlCheck) {
    pbf::block_partial<kBlock>(err, io.partials + blockIdx.x);
    pbf::decide_if_last<kBlock, LOOP>(io.state, io.partials, n, io.tol, io.final_check, io.loop);
  }
}

// The learned solver's sampled residual check (residual_sample = S > 1): the
// density of every S-th run of kProbeRun consecutive sorted slots over its
// list (runs keep the gathers' neighbour records shared, as in the full pass),
// the mean clamped error of those particles decided as kDlCheck does
// (pbf::decide_if_last over the samples); nothing else is written.  The nudge
// of a coincident neighbour is left out of the estimate.
constexpr int kProbeRun = 32;

template <int GL, bool LOOP>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) kl_residual_probe(Dev P, Fast F, int n, int stride_s,
                                                                              size_t stride,
                                                                              const int32_t* __restrict__ nbr,
                                                                              const int32_t* __restrict__ cnt,
                                                                              const float4* __restrict__ pst,
                                                                              LearnIO io) {
  if (io.state->done) {
    if constexpr (LOOP)
      if (io.loop.use && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(io.loop.cond, 0u);
    return;
  }
  const int span = kProbeRun * stride_s;  // one run sampled per span of slots
  const int runs = (n + span - 1) / span;
  const int ns = runs * kProbeRun;        // sample k: slot (k / run) * span + k % run, live below n
  const int last = n - (runs - 1) * span;
  const int live = (runs - 1) * kProbeRun + (last < kProbeRun ? last : kProbeRun);
  const int tiles = pbf::tiles_of<GL>(ns);
  float err = 0.0f;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    pbf::Group G = pbf::group_at<GL>(ns, tile);
    const int slot = (G.b / kProbeRun) * span + G.b % kProbeRun;
    G.live = G.live && slot < n;
    G.b = G.live ? slot : 0;
    const int b = G.b;
    const float4 xp = pst[b];
    const int c = G.live ? cnt[b] : 0;
    const DensitySums S = density_sums<GL, false>(F, G, nbr + pbf::list_base(b, stride), nullptr, c, n, pst, xp);
    if (G.live && G.lane == 0) err += fmaxf(fmaf(fmaf(F.m_poly, S.sw, F.m_w0), F.inv_rho0, -1.0f), 0.0f);
  }
  pbf::block_partial<kBlock>(err, io.partials + blockIdx.x);
  pbf::decide_if_last<kBlock, LOOP>(io.state, io.partials, live, io.tol, io.final_check, io.loop);
}

// ---- staged gathers: one 32-particle tile per block of kStageThreads ----
constexpr int kStageThreads = kTile * 4;  // 4 lanes per particle

// Copy the tile's neighbour records (the runs of its descriptor) from a (and
// b2 when B2) to shared memory, the zero record after them; every thread of
// the block calls it.  Returns the staged count, or -1 for a tile the list
// fill did not stage (its gathers then walk the int32 lists).
template <bool B2>
__device__ __forceinline__ int stage_tile(const TileIO& T, int tile, const float4* __restrict__ a, float4* sa,
                                          const float4* __restrict__ b2, float4* sb) {
  __shared__ int4 runs[kTileRuns];
  __shared__ int hdr[2];
  if (threadIdx.x < kTileRuns) runs[threadIdx.x] = T.runs[(size_t)tile * kTileRuns + threadIdx.x];
  if (threadIdx.x == 0) {
    hdr[0] = T.nruns[tile];
    hdr[1] = T.total[tile];
  }
  __syncthreads();
  const int nr = hdr[0], total = hdr[1];
  if (nr > 0) {
    for (int r = 0; r < nr; ++r) {
      const int4 ru = runs[r];
      for (int i = threadIdx.x; i < ru.y; i += blockDim.x) {
        sa[ru.z + i] = a[ru.x + i];
        if (B2) sb[ru.z + i] = b2[ru.x + i];
      }
    }
    if (threadIdx.x == 0) {
      sa[total] = make_float4(kFar, kFar, kFar, 0.0f);
      if (B2) sb[total] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    }
  }
  __syncthreads();
  return nr > 0 ? total : -1;
}

template <int MODE, bool LOOP = false>
__global__ void __launch_bounds__(kStageThreads) ks_density_lambda(Dev P, Fast F, int n, size_t stride,
                                                                  const int32_t* __restrict__ nbr,
                                                                  const int32_t* __restrict__ cnt,
                                                                  const float4* __restrict__ pst, float4* xl,
                                                                  float4* vel, float* lam, uint32_t* nudge, LearnIO io,
                                                                  TileIO T) {
  __shared__ float4 stage[kStageMax + 1];
  if (MODE == kDlCheck && io.state->done) {
    if constexpr (LOOP)
      if (io.loop.use && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(io.loop.cond, 0u);
    return;
  }
  const int tiles = (n + kTile - 1) / kTile;
  float err = 0.0f;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int staged = stage_tile<false>(T, tile, pst, stage, nullptr, nullptr);
    if (staged >= 0)
      density_lambda_tile<MODE, 4, true>(tile, P, F, n, stride, nbr, cnt, pst, xl, vel, lam, nudge, io, err, T.nbr16,
                                         stage, staged);
    else
      density_lambda_tile<MODE, 4>(tile, P, F, n, stride, nbr, cnt, pst, xl, vel, lam, nudge, io, err);
    __syncthreads();  // the next tile's staging overwrites the area
  }
  if (MODE == kDlCheck) {
    pbf::block_partial<kStageThreads>(err, io.partials + blockIdx.x);
    pbf::decide_if_last<kStageThreads, LOOP>(io.state, io.partials, n, io.tol, io.final_check, io.loop);
  }
}

// Learned warm start, first Jacobi iteration, in two launches:
// kl_features: the gather of kf_density_lambda, then per particle the 12
// normalised features as a BF16 row of 16 (columns 12..15 are padding the
// network's first layer multiplies by zero; column 15 flags a particle the
// reference-ordered nudge path handled), and the plain first-iteration
// lambda l1 in xl.w.
// kl_mlp_tc<true>: the network on the tensor cores (tcgen05, below);
// lambda = the output kept between l1 and kWarmMaxGain * l1.
// A single over-relaxed iteration on its own overshoots and the overshoot
// feeds the velocity update (measured on the oracle: 1 iteration at 2.5x
// lambda ends near 4% density error where 1 plain iteration ends near 1.5%),
// so the residual-checked plain iterations that follow are part of the method.
// The bound 5 was chosen on a validation trajectory (1M dam, relaxation
// epsilon 1, seed 5151, steps 100-140): 1.98 / 1.86 / 1.84 / 1.86 ms per
// step at 3 / 4 / 5 / 6 (2.8 / 2.55 / 2.35 / 2.5 iterations).
constexpr float kWarmMaxGain = 5.0f;

template <int GL>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) kl_features(Dev P, Fast F, pbf::MlpDev M, int n,
                                                                        size_t stride,
                                                      const int32_t* __restrict__ nbr, const int32_t* __restrict__ cnt,
                                                      const float4* __restrict__ pst, float4* xl, float4* vel,
                                                      float* lam, uint32_t* nudge, const float* __restrict__ lamprev,
                                                      __nv_bfloat16* featb) {
  const pbf::Group G = pbf::group_of<GL>(n);
  const int b = G.b;
  const float4 xp = pst[b];
  const int c = G.live ? cnt[b] : 0;
  const DensitySums S = density_sums<GL, true>(F, G, nbr + pbf::list_base(b, stride), nullptr, c, n, pst, xp);
  if (!G.live || G.lane != 0) return;
  const float rho = fmaf(F.m_poly, S.sw, F.m_w0);
  const float L2 = F.lam_grad * F.lam_grad;
  const float sc = L2 * S.s2;
  const float g2 = L2 * fmaf(S.s1z, S.s1z, fmaf(S.s1y, S.s1y, S.s1x * S.s1x));
  const bool close = S.dmin < 4e-16f;
  const float nh = S.nh;
  const float4 v = vel[b];
  float f[pbf::kMlpIn];
  pbf::raw_features(P, pbf::region_of(P, b), F, f, c, rho, sc, g2, (int)nh, lamprev[b], v, xp);
  uint32_t row[pbf::kMlpInPad / 2];
#pragma unroll
  for (int k = 0; k < pbf::kMlpIn; k += 2)
    row[k / 2] = pbf::pack_bf16x2((f[k] - M.feat_mean[k]) * M.feat_inv_std[k],
                                  (f[k + 1] - M.feat_mean[k + 1]) * M.feat_inv_std[k + 1]);
  row[6] = 0u;
  row[7] = pbf::pack_bf16x2(0.0f, close ? 1.0f : 0.0f);
  uint4* dst = reinterpret_cast<uint4*>(featb + (size_t)b * pbf::kMlpInPad);
  dst[0] = make_uint4(row[0], row[1], row[2], row[3]);
  dst[1] = make_uint4(row[4], row[5], row[6], row[7]);
  if (close) {
    density_lambda_one<false>(P, b, stride, nbr, cnt, pst, xl, vel, lam, nudge);
    return;
  }
  const float C = fmaxf(fmaf(rho, F.inv_rho0, -1.0f), 0.0f);
  const float l1 = -C / (sc + g2 + F.lambda_eps);
  xl[b] = make_float4(xp.x, xp.y, xp.z, l1);
  vel[b] = make_float4(v.x, v.y, v.z, rho);
  lam[b] = l1;
}

// The network on the 5th-generation tensor cores (see pbf_mlp_tc.cuh): a
// persistent grid of 256-thread CTAs, each holding the weights in shared
// memory and 64 TMEM columns, walking 128-row tiles.  Two threads per row
// (warps w and w + 4 read the same TMEM lanes), each for 32 of the 64 hidden
// columns.  Per tile: the rows' BF16 features -> one M128 N64 K16 MMA ->
// layer-1 epilogue (bias, GELU, BF16 back to shared memory as layer 2's A
// operand) -> four M128 N64 K16 MMAs into the same columns -> layer-2
// epilogue (bias, GELU, the dot with w3, the two halves added).
// WARM: features from featb (column 15 flags the reference-ordered nudge
// path), lambda = the output kept between l1 and kWarmMaxGain * l1.
// PREDICT: normalised float features, y = the output.  A wait that gives up
// raises PBF_FLAG_WAIT_TIMEOUT; every CTA frees its TMEM.
// NO_ARRIVE (the failure-path self-test only): the MMAs and their commits
// are left out, so nothing arrives on the barrier and every bounded wait runs
// out; nothing asynchronous is in flight when the kernel gives up.
template <bool WARM, bool NO_ARRIVE = false>
__global__ void __launch_bounds__(pbf::tc::kThreads, 6) kl_mlp_tc(pbf::MlpDev M, int n,
                                                              const __nv_bfloat16* __restrict__ featb,
                                                              const float* __restrict__ feats, float4* xl,
                                                              float* lam, float* lamsum, float* y, uint32_t* err) {
  namespace T = pbf::tc;
  __shared__ __align__(1024) uint8_t sB1[pbf::kMlpH * pbf::kMlpInPad * 2];  // W1 [64 n][16 k]
  __shared__ __align__(1024) uint8_t sB2[pbf::kMlpH * pbf::kMlpH * 2];      // W2 [64 n][64 k]
  __shared__ __align__(1024) uint8_t sA1[T::kRows * pbf::kMlpInPad * 2];    // features [128][16]
  __shared__ __align__(1024) uint8_t sA2[T::kRows * pbf::kMlpH * 2];        // hidden 1 [128][64]
  __shared__ __align__(16) float sb1[pbf::kMlpH];  // read as float2 pairs
  __shared__ __align__(16) float sb2[pbf::kMlpH];
  __shared__ __align__(16) float sw3[pbf::kMlpH];
  __shared__ float half2[T::kRows];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ int fail;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int row = tid & (T::kRows - 1), h = tid >> 7;  // row in the tile, column half
  const int tiles = (n + T::kRows - 1) / T::kRows;
  for (int i = tid; i < pbf::kMlpH * 2; i += T::kThreads) {  // W1: 64 rows x 2 chunks of 8 along k
    const int r = i >> 1, kc = (i & 1) * 8;
    *reinterpret_cast<uint4*>(sB1 + T::core_off(r, kc, pbf::kMlpInPad)) =
        *reinterpret_cast<const uint4*>(M.w1 + r * pbf::kMlpInPad + kc);
  }
  for (int i = tid; i < pbf::kMlpH * 8; i += T::kThreads) {  // W2: 64 rows x 8 chunks
    const int r = i >> 3, kc = (i & 7) * 8;
    *reinterpret_cast<uint4*>(sB2 + T::core_off(r, kc, pbf::kMlpH)) =
        *reinterpret_cast<const uint4*>(M.w2 + r * pbf::kMlpH + kc);
  }
  if (tid < pbf::kMlpH) {
    sb1[tid] = M.b1[tid];
    sb2[tid] = M.b2[tid];
    sw3[tid] = M.w3[tid];
  }
  const uint32_t bar = T::smem_u32(&mbar);
  if (tid == 0) {
    T::bar_init(bar, 1);
    fail = 0;
  }
  if (warp == 0) T::tmem_alloc(T::smem_u32(&tslot));
  T::fence_before_sync();
  __syncthreads();
  T::fence_after_sync();
  const uint32_t tmem = tslot;
  const uint32_t lanes = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(32 * h);  // this thread's half
  const float b3 = M.b3[0];
  const uint64_t dB1 = T::smem_desc(T::smem_u32(sB1), 128, 256);
  const uint32_t a1 = T::smem_u32(sA1), a2 = T::smem_u32(sA2), b2 = T::smem_u32(sB2);
  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int r = tile * T::kRows + row;
    uint4 f = make_uint4(0u, 0u, 0u, 0u);  // half h of the row's 16 features
    if (r < n) {
      if (WARM) {
        f = reinterpret_cast<const uint4*>(featb + (size_t)r * pbf::kMlpInPad)[h];
      } else if (h == 0) {
        const float* x = feats + (size_t)r * pbf::kMlpIn;
        f = make_uint4(pbf::pack_bf16x2(x[0], x[1]), pbf::pack_bf16x2(x[2], x[3]), pbf::pack_bf16x2(x[4], x[5]),
                       pbf::pack_bf16x2(x[6], x[7]));
      } else {
        const float* x = feats + (size_t)r * pbf::kMlpIn;
        f = make_uint4(pbf::pack_bf16x2(x[8], x[9]), pbf::pack_bf16x2(x[10], x[11]), 0u, 0u);
      }
    }
    const uint32_t flag = f.w >> 16;  // h = 1: column 15 (WARM: the nudge path handled the particle)
    // columns 12..15 meet zero rows of W1; the flag column is cleared for the MMA
    *reinterpret_cast<uint4*>(sA1 + T::core_off(row, 8 * h, pbf::kMlpInPad)) =
        h ? make_uint4(f.x, f.y, 0u, 0u) : f;
    T::fence_proxy_async();
    T::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      T::fence_after_sync();
      if (!NO_ARRIVE) {
        T::mma_bf16(tmem, T::smem_desc(a1, 128, 256), dB1, T::kIdescM128N64, 0u);
        T::mma_commit(bar);
      }
    }
    if (!T::bar_wait(bar, phase)) fail = 1;
    phase ^= 1u;
    __syncthreads();
    if (fail) break;
    T::fence_after_sync();
#pragma unroll
    for (int c = 0; c < 32; c += 16) {
      float v[16];
      T::tmem_ld16(lanes + (uint32_t)c, v);
      const int c0 = 32 * h + c;
#pragma unroll
      for (int j = 0; j < 16; j += 8) {
        uint32_t wq[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float2 b = *reinterpret_cast<const float2*>(sb1 + c0 + j + 2 * k);
          const float2 g = pbf::gelu2(__fadd2_rn(make_float2(v[j + 2 * k], v[j + 2 * k + 1]), b));
          wq[k] = pbf::pack_bf16x2(g.x, g.y);
        }
        *reinterpret_cast<uint4*>(sA2 + T::core_off(row, c0 + j, pbf::kMlpH)) = make_uint4(wq[0], wq[1], wq[2], wq[3]);
      }
    }
    T::fence_proxy_async();
    T::fence_before_sync();
    __syncthreads();  // every layer-1 accumulator read before layer 2 overwrites them
    if (tid == 0) {
      T::fence_after_sync();
      if (!NO_ARRIVE) {
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)
          T::mma_bf16(tmem, T::smem_desc(a2 + 256u * ks, 128, 1024), T::smem_desc(b2 + 256u * ks, 128, 1024),
                      T::kIdescM128N64, ks > 0 ? 1u : 0u);
        T::mma_commit(bar);
      }
    }
    if (!T::bar_wait(bar, phase)) fail = 1;
    phase ^= 1u;
    __syncthreads();
    if (fail) break;
    T::fence_after_sync();
    float2 acc2 = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int c = 0; c < 32; c += 16) {
      float v[16];
      T::tmem_ld16(lanes + (uint32_t)c, v);
      const int c0 = 32 * h + c;
#pragma unroll
      for (int q = 0; q < 16; q += 2) {
        const float2 b = *reinterpret_cast<const float2*>(sb2 + c0 + q);
        const float2 w3 = *reinterpret_cast<const float2*>(sw3 + c0 + q);
        acc2 = __ffma2_rn(pbf::gelu2(__fadd2_rn(make_float2(v[q], v[q + 1]), b)), w3, acc2);
      }
    }
    const float acc = acc2.x + acc2.y;
    if (h == 0) half2[row] = acc;
    T::fence_before_sync();
    __syncthreads();  // the first halves in shared memory; TMEM and operands free for the next tile
    if (h == 1 && r < n) {
      const float yv = half2[row] + acc + b3;
      if (WARM) {
        const float4 x = xl[r];
        float l = x.w;  // l1, or the nudge path's lambda
        if (flag == 0u) l = fminf(fmaxf(yv * M.label_scale, kWarmMaxGain * x.w), x.w);
        xl[r] = make_float4(x.x, x.y, x.z, l);
        lam[r] = l;
        lamsum[r] = l;
      } else {
        y[r] = yv;
      }
    }
  }
  if (fail && tid == 0) atomicOr(err, PBF_FLAG_WAIT_TIMEOUT);
  __syncthreads();
  if (warp == 0) {
    T::fence_after_sync();
    T::tmem_free(tmem);
  }
}

// Lambda recomputed from the (nudged) positions in xl, only when the
// preceding density_lambda launch nudged a particle; otherwise every block
// returns at once.
template <bool X>
__global__ void __launch_bounds__(kBlock) k_lambda_fixup(Dev P, int n, size_t stride, const int32_t* __restrict__ nbr,
                                                         const int32_t* __restrict__ cnt,
                                                         const float4* __restrict__ xl, const float4* __restrict__ vel,
                                                         float* lam, const uint32_t* __restrict__ nudge) {
  if (*nudge == 0u) return;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const float4 xp = xl[b];
  const int c = cnt[b];
  float3 sg = make_float3(0.f, 0.f, 0.f);
  float sumC = 0.0f;
  for (int k = 0; k < c; ++k) {
    const float4 xq = xl[nbr[pbf::list_at(b, stride, k)]];
    const float rx = pbf::S<X>(xp.x, xq.x), ry = pbf::S<X>(xp.y, xq.y), rz = pbf::S<X>(xp.z, xq.z);
    lambda_terms<X>(P, rx, ry, rz, pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz)), sg, sumC);
  }
  lam[b] = lambda_of<X>(P, vel[b].w, sg, sumC);
}

// compute_pressure_dps (particles.h:348-358) summand; s_corr optional.
template <bool X, bool SCORR>
__device__ __forceinline__ void dp_term(const Dev& P, float lp, float lq, float rx, float ry, float rz, float rm,
                                        float3& dp) {
  float l = pbf::A<X>(lp, lq);
  if (SCORR) {
    const float w = pbf::poly6<X>(P, rm);
    l = l - P.scorr_k * powf(w * P.inv_wdq, P.scorr_n);
  }
  const float3 dw = pbf::del_spikey<X>(P, rx, ry, rz, rm);
  dp.x = pbf::A<X>(dp.x, pbf::M<X>(l, dw.x));
  dp.y = pbf::A<X>(dp.y, pbf::M<X>(l, dw.y));
  dp.z = pbf::A<X>(dp.z, pbf::M<X>(l, dw.z));
}

// Per-stage delta-p -> scratch.
template <bool X, bool SCORR>
__global__ void __launch_bounds__(kBlock) k_dp(Dev P, int n, size_t stride, const int32_t* __restrict__ nbr,
                                               const int32_t* __restrict__ cnt, const float4* __restrict__ pst,
                                               const float* __restrict__ lam, float4* scr) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n || !pbf::in_span(P, b)) return;
  const float4 xp = pst[b];
  const float lp = lam[b];
  const int c = cnt[b];
  float3 dp = make_float3(0.f, 0.f, 0.f);
  for (int k = 0; k < c; ++k) {
    const int q = nbr[pbf::list_at(b, stride, k)];
    const float4 xq = pst[q];
    const float rx = pbf::S<X>(xp.x, xq.x), ry = pbf::S<X>(xp.y, xq.y), rz = pbf::S<X>(xp.z, xq.z);
    dp_term<X, SCORR>(P, lp, lam[q], rx, ry, rz, pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz)), dp);
  }
  scr[b] = make_float4(pbf::M<X>(P.inv_rho0, dp.x), pbf::M<X>(P.inv_rho0, dp.y), pbf::M<X>(P.inv_rho0, dp.z), 0.0f);
}

// update_position_stars (particles.h:363-370), per-stage.
__global__ void k_update_xs(Dev P, int n, float4* pst, const float4* __restrict__ scr) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n || !pbf::in_span(P, b)) return;
  const float4 x = pst[b], d = scr[b];
  const float3 s = pbf::boundary(P, pbf::region_of(P, b),
                                 make_float3(pbf::xadd(x.x, d.x), pbf::xadd(x.y, d.y), pbf::xadd(x.z, d.z)));
  pst[b] = make_float4(s.x, s.y, s.z, 0.0f);
}

// update_velocities (particles.h:375-385), always exact (per-particle).
__device__ __forceinline__ float3 velocity_of(const Dev& P, float4 xs, float4 x) {
  float3 v = make_float3(pbf::xdiv(pbf::xsub(xs.x, x.x), P.dt), pbf::xdiv(pbf::xsub(xs.y, x.y), P.dt),
                         pbf::xdiv(pbf::xsub(xs.z, x.z), P.dt));
  if ((double)pbf::mag2<true>(v.x, v.y, v.z) < P.vthr) v = make_float3(0.f, 0.f, 0.f);
  return v;
}

__global__ void k_update_v(Dev P, int n, const float4* __restrict__ pst, const float4* __restrict__ pos,
                           float4* vel) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n || !pbf::in_span(P, b)) return;
  const float3 v = velocity_of(P, pst[b], pos[b]);
  vel[b] = make_float4(v.x, v.y, v.z, vel[b].w);
}

// update_positions (particles.h:390-394) over a span: x = x* inside it.
__global__ void k_update_positions(Dev P, int n, const float4* __restrict__ pst, float4* pos) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n || !pbf::in_span(P, b)) return;
  pos[b] = pst[b];
}

// Empty neighbor lists for the particles outside a fill span.
__global__ void k_clear_outside_span(int n, const uint32_t* __restrict__ orig, uint32_t end, int32_t* cnt) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n && orig[b] >= end) cnt[b] = 0;
}

// Fused delta-p + x* update (+ velocity update on the last iteration): reads
// (x*, lambda) of neighbours from xl, writes the new x* (Jacobi: nobody reads
// pst in this kernel).
template <bool X, bool SCORR, bool LAST>
__global__ void __launch_bounds__(kBlock) k_dp_update(Dev P, int n, size_t stride, const int32_t* __restrict__ nbr,
                                                      const int32_t* __restrict__ cnt, const float4* __restrict__ xl,
                                                      float4* pst, const float4* __restrict__ pos, float4* vel,
                                                      const float* __restrict__ lam,
                                                      const uint32_t* __restrict__ nudge) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const float4 xp = xl[b];
  const int c = cnt[b];
  float3 dp = make_float3(0.f, 0.f, 0.f);
  if (*nudge == 0u) {
    for (int k = 0; k < c; ++k) {
      const float4 xq = xl[nbr[pbf::list_at(b, stride, k)]];
      const float rx = pbf::S<X>(xp.x, xq.x), ry = pbf::S<X>(xp.y, xq.y), rz = pbf::S<X>(xp.z, xq.z);
      dp_term<X, SCORR>(P, xp.w, xq.w, rx, ry, rz, pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz)), dp);
    }
  } else {  // lambdas were recomputed by k_lambda_fixup
    const float lp = lam[b];
    for (int k = 0; k < c; ++k) {
      const int q = nbr[pbf::list_at(b, stride, k)];
      const float4 xq = xl[q];
      const float rx = pbf::S<X>(xp.x, xq.x), ry = pbf::S<X>(xp.y, xq.y), rz = pbf::S<X>(xp.z, xq.z);
      dp_term<X, SCORR>(P, lp, lam[q], rx, ry, rz, pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz)), dp);
    }
  }
  const float dx = pbf::M<X>(P.inv_rho0, dp.x), dy = pbf::M<X>(P.inv_rho0, dp.y), dz = pbf::M<X>(P.inv_rho0, dp.z);
  const float3 s = pbf::boundary(P, pbf::region_of(P, b),
                                 make_float3(pbf::xadd(xp.x, dx), pbf::xadd(xp.y, dy), pbf::xadd(xp.z, dz)));
  const float4 ns = make_float4(s.x, s.y, s.z, 0.0f);
  pst[b] = ns;
  if (LAST) {
    const float3 v = velocity_of(P, ns, pos[b]);
    vel[b] = make_float4(v.x, v.y, v.z, vel[b].w);
  }
}

// apply_surface_tension (particles.h:400-431): colour-field pass ...
template <bool X>
__global__ void __launch_bounds__(kBlock) k_color(Dev P, int n, size_t stride, const int32_t* __restrict__ nbr,
                                                  const int32_t* __restrict__ cnt, const float4* __restrict__ pst,
                                                  const float4* __restrict__ vel, float4* scr) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n || !pbf::in_span(P, b)) return;
  const float4 xp = pst[b];
  const int c = cnt[b];
  float3 col = make_float3(0.f, 0.f, 0.f);
  for (int k = 0; k < c; ++k) {
    const int q = nbr[pbf::list_at(b, stride, k)];
    const float4 xq = pst[q];
    const float rq = vel[q].w;
    const float rx = pbf::S<X>(xp.x, xq.x), ry = pbf::S<X>(xp.y, xq.y), rz = pbf::S<X>(xp.z, xq.z);
    const float3 dw = pbf::del_spikey<X>(P, rx, ry, rz, pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz)));
    col.x = pbf::A<X>(col.x, pbf::D<X>(dw.x, rq));
    col.y = pbf::A<X>(col.y, pbf::D<X>(dw.y, rq));
    col.z = pbf::A<X>(col.z, pbf::D<X>(dw.z, rq));
  }
  scr[b] = make_float4(pbf::M<X>(P.h, col.x), pbf::M<X>(P.h, col.y), pbf::M<X>(P.h, col.z), 0.0f);
}

// ... then the cohesion + curvature force pass (always exact: rare path).
__global__ void __launch_bounds__(kBlock) k_surface(Dev P, int n, size_t stride, const int32_t* __restrict__ nbr,
                                                    const int32_t* __restrict__ cnt, const float4* __restrict__ pst,
                                                    const float4* __restrict__ scr, float4* vel) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n || !pbf::in_span(P, b)) return;
  const float4 xp = pst[b], sp = scr[b];
  const float rp = vel[b].w;
  const int c = cnt[b];
  const float ng = -P.gamma;
  float3 f = make_float3(0.f, 0.f, 0.f);
  for (int k = 0; k < c; ++k) {
    const int q = nbr[pbf::list_at(b, stride, k)];
    const float4 xq = pst[q], sq = scr[q];
    const float rq = vel[q].w;
    const float rx = pbf::xsub(xp.x, xq.x), ry = pbf::xsub(xp.y, xq.y), rz = pbf::xsub(xp.z, xq.z);
    float rm = __fsqrt_rn(pbf::mag2<true>(rx, ry, rz));
    if ((double)rm < P.h_eps) rm = (float)P.h_eps;
    const float cs = pbf::xmul(ng, pbf::c_spline<true>(P, rm));
    const float K = (float)__ddiv_rn(__dmul_rn(2.0, (double)P.rho0), (double)pbf::xadd(rp, rq));
    f.x = pbf::xadd(f.x, pbf::xmul(K, pbf::xadd(pbf::xdiv(pbf::xmul(cs, rx), rm), pbf::xmul(ng, pbf::xsub(sp.x, sq.x)))));
    f.y = pbf::xadd(f.y, pbf::xmul(K, pbf::xadd(pbf::xdiv(pbf::xmul(cs, ry), rm), pbf::xmul(ng, pbf::xsub(sp.y, sq.y)))));
    f.z = pbf::xadd(f.z, pbf::xmul(K, pbf::xadd(pbf::xdiv(pbf::xmul(cs, rz), rm), pbf::xmul(ng, pbf::xsub(sp.z, sq.z)))));
  }
  float4 v = vel[b];
  v.x = pbf::xadd(v.x, pbf::xmul(pbf::xdiv(f.x, rp), P.dt));
  v.y = pbf::xadd(v.y, pbf::xmul(pbf::xdiv(f.y, rp), P.dt));
  v.z = pbf::xadd(v.z, pbf::xmul(pbf::xdiv(f.z, rp), P.dt));
  vel[b] = v;
}

// XSPH viscosity (particles.h:436-447), Jacobi: reads vin, writes vout.
// FINAL also performs update_positions (particles.h:390-394) and writes the
// step's results into the home buffers.
template <bool X, bool FINAL>
__global__ void __launch_bounds__(kBlock) k_viscosity(Dev P, int n, size_t stride, const int32_t* __restrict__ nbr,
                                                      const int32_t* __restrict__ cnt, const float4* __restrict__ pst,
                                                      const float4* __restrict__ vin, float4* vout, float4* posH,
                                                      float4* pstH, const uint32_t* __restrict__ origS,
                                                      uint32_t* origH) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const float4 xp = pst[b], vp = vin[b];
  if (!FINAL && !pbf::in_span(P, b)) {  // outside the span: v stays
    vout[b] = vp;
    return;
  }
  const int c = cnt[b];
  float3 dv = make_float3(0.f, 0.f, 0.f);
  for (int k = 0; k < c; ++k) {
    const int q = nbr[pbf::list_at(b, stride, k)];
    const float4 xq = pst[q], vq = vin[q];
    const float rx = pbf::S<X>(xp.x, xq.x), ry = pbf::S<X>(xp.y, xq.y), rz = pbf::S<X>(xp.z, xq.z);
    const float w = pbf::poly6<X>(P, pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz)));
    if (X) {
      dv.x = pbf::xadd(dv.x, pbf::xdiv(pbf::xmul(pbf::xsub(vq.x, vp.x), w), vq.w));
      dv.y = pbf::xadd(dv.y, pbf::xdiv(pbf::xmul(pbf::xsub(vq.y, vp.y), w), vq.w));
      dv.z = pbf::xadd(dv.z, pbf::xdiv(pbf::xmul(pbf::xsub(vq.z, vp.z), w), vq.w));
    } else {
      const float wr = __fdividef(w, vq.w);
      dv.x = fmaf(vq.x - vp.x, wr, dv.x);
      dv.y = fmaf(vq.y - vp.y, wr, dv.y);
      dv.z = fmaf(vq.z - vp.z, wr, dv.z);
    }
  }
  vout[b] = make_float4(pbf::A<X>(vp.x, pbf::M<X>(P.visc_c, dv.x)), pbf::A<X>(vp.y, pbf::M<X>(P.visc_c, dv.y)),
                        pbf::A<X>(vp.z, pbf::M<X>(P.visc_c, dv.z)), vp.w);
  if (FINAL) {
    posH[b] = xp;
    pstH[b] = xp;
    origH[b] = origS[b];
  }
}

// compute_vorticity (particles.h:452-466): omega into scratch (w = |omega|,
// computed as magnitude() would) and (x*, |omega|) into xl for the apply pass.
template <bool X>
__global__ void __launch_bounds__(kBlock) k_vorticity(Dev P, int n, size_t stride, const int32_t* __restrict__ nbr,
                                                      const int32_t* __restrict__ cnt, const float4* __restrict__ pst,
                                                      const float4* __restrict__ vel, float4* scr, float4* xl) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n || !pbf::in_span(P, b)) return;
  const float4 xp = pst[b], vp = vel[b];
  const int c = cnt[b];
  float3 w = make_float3(0.f, 0.f, 0.f);
  for (int k = 0; k < c; ++k) {
    const int q = nbr[pbf::list_at(b, stride, k)];
    const float4 xq = pst[q], vq = vel[q];
    const float rx = pbf::S<X>(xp.x, xq.x), ry = pbf::S<X>(xp.y, xq.y), rz = pbf::S<X>(xp.z, xq.z);
    const float3 d = pbf::del_spikey<X>(P, rx, ry, rz, pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz)));
    const float ax = pbf::S<X>(vq.x, vp.x), ay = pbf::S<X>(vq.y, vp.y), az = pbf::S<X>(vq.z, vp.z);
    // cross(v_diff, del) (vec.h:622-630)
    w.x = pbf::A<X>(w.x, pbf::S<X>(pbf::M<X>(ay, d.z), pbf::M<X>(az, d.y)));
    w.y = pbf::A<X>(w.y, pbf::S<X>(pbf::M<X>(az, d.x), pbf::M<X>(ax, d.z)));
    w.z = pbf::A<X>(w.z, pbf::S<X>(pbf::M<X>(ax, d.y), pbf::M<X>(ay, d.x)));
  }
  const float wm = __fsqrt_rn(pbf::mag2<true>(w.x, w.y, w.z));
  scr[b] = make_float4(w.x, w.y, w.z, wm);
  if (xl) xl[b] = make_float4(xp.x, xp.y, xp.z, wm);
}

// apply_vorticity (particles.h:471-487).  PACKED reads (x*, |omega|) of
// neighbours from xl (one 16-byte load); otherwise from pst and scratch.
template <bool X, bool PACKED>
__global__ void __launch_bounds__(kBlock) k_apply_vorticity(Dev P, int n, size_t stride,
                                                            const int32_t* __restrict__ nbr,
                                                            const int32_t* __restrict__ cnt,
                                                            const float4* __restrict__ xl,
                                                            const float4* __restrict__ pst,
                                                            const float4* __restrict__ scr, float4* vel) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n || !pbf::in_span(P, b)) return;
  const float4 xp = PACKED ? xl[b] : pst[b];
  const int c = cnt[b];
  float3 eta = make_float3(0.f, 0.f, 0.f);
  for (int k = 0; k < c; ++k) {
    const int q = nbr[pbf::list_at(b, stride, k)];
    float4 xq;
    float vm;
    if (PACKED) {
      xq = xl[q];
      vm = xq.w;
    } else {
      xq = pst[q];
      const float4 sq = scr[q];
      vm = __fsqrt_rn(pbf::mag2<true>(sq.x, sq.y, sq.z));
    }
    const float rx = pbf::S<X>(xp.x, xq.x), ry = pbf::S<X>(xp.y, xq.y), rz = pbf::S<X>(xp.z, xq.z);
    const float3 d = pbf::del_spikey<X>(P, rx, ry, rz, pbf::SQ<X>(pbf::mag2<X>(rx, ry, rz)));
    eta.x = pbf::A<X>(eta.x, pbf::M<X>(vm, d.x));
    eta.y = pbf::A<X>(eta.y, pbf::M<X>(vm, d.y));
    eta.z = pbf::A<X>(eta.z, pbf::M<X>(vm, d.z));
  }
  const float den = pbf::A<X>(pbf::SQ<X>(pbf::mag2<X>(eta.x, eta.y, eta.z)), FLT_EPSILON);
  const float Nx = pbf::D<X>(eta.x, den), Ny = pbf::D<X>(eta.y, den), Nz = pbf::D<X>(eta.z, den);
  const float4 wp = scr[b];
  const float cx = pbf::S<X>(pbf::M<X>(Ny, wp.z), pbf::M<X>(Nz, wp.y));
  const float cy = pbf::S<X>(pbf::M<X>(Nz, wp.x), pbf::M<X>(Nx, wp.z));
  const float cz = pbf::S<X>(pbf::M<X>(Nx, wp.y), pbf::M<X>(Ny, wp.x));
  float4 v = vel[b];
  v.x = pbf::A<X>(v.x, pbf::M<X>(pbf::M<X>(cx, P.vort_eps), P.dt));
  v.y = pbf::A<X>(v.y, pbf::M<X>(pbf::M<X>(cy, P.vort_eps), P.dt));
  v.z = pbf::A<X>(v.z, pbf::M<X>(pbf::M<X>(cz, P.vort_eps), P.dt));
  vel[b] = v;
}

// ---- fast gathers (exact_math = 0), kGL lanes per particle, see pbf_fast.cuh ----
// COND: the learned solver's extra iterations, skipped once the step has
// converged; lamsum (when given) accumulates the applied lambda.
// Where a gather's neighbour records come from: the tile's staging area
// (STAGED: shared memory through the 16-bit list) or global memory.
struct Src {
  const uint16_t* nbr16;  // STAGED: the 16-bit lists
  const float4* a;        // first record array (staged copy or global)
  const float4* b;        // second record array (two-record gathers)
  int dummy;              // index of the zero record
};

template <bool SCORR, bool LAST, int GL, bool STAGED = false, bool COH = false>
__device__ __forceinline__ void dp_update_tile(int tile, const Dev& P, const Fast& F, int n, size_t stride,
                                               const int32_t* __restrict__ nbr, const int32_t* __restrict__ cnt,
                                               const float4* __restrict__ xl, float4* pst,
                                               const float4* __restrict__ pos, float4* vel, float* lamsum,
                                               Src src = Src{nullptr, nullptr, nullptr, 0}) {
  const pbf::Group G = pbf::group_at<GL>(n, tile);
  const int b = G.b;
  const float4 xp = xl[b];
  const int c = G.live ? cnt[b] : 0;
  float ax = 0.f, ay = 0.f, az = 0.f;
  const float lp = xp.w;
  pbf::walk1<GL, STAGED, false, COH>(nbr + pbf::list_base(b, stride),
                                     STAGED ? src.nbr16 + (size_t)b * stride : nullptr, c, STAGED ? src.dummy : n,
                                     G.lane, STAGED ? src.a : xl, [&](int, float4 xq) {
    const float dx = xp.x - xq.x, dy = xp.y - xq.y, dz = xp.z - xq.z;
    const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    float l = lp + xq.w;
    if (SCORR) l -= P.scorr_k * __powf(F.visc_poly * pbf::poly_cube(F, d2) * P.inv_wdq, P.scorr_n);
    const float t = l * pbf::spikey_over_r(F, d2);
    ax = fmaf(t, dx, ax);
    ay = fmaf(t, dy, ay);
    az = fmaf(t, dz, az);
  });
  ax = pbf::gsum<GL>(ax);
  ay = pbf::gsum<GL>(ay);
  az = pbf::gsum<GL>(az);
  if (!G.live || G.lane != 0) return;
  if (lamsum) lamsum[b] += xp.w;
  const float3 s = pbf::boundary(P, pbf::region_of(P, b),
                                 make_float3(pbf::xadd(xp.x, F.dp_scale * ax), pbf::xadd(xp.y, F.dp_scale * ay),
                                                pbf::xadd(xp.z, F.dp_scale * az)));
  const float4 ns = make_float4(s.x, s.y, s.z, 0.0f);
  pst[b] = ns;
  if (LAST) {
    const float3 v = velocity_of(P, ns, pos[b]);
    vel[b] = make_float4(v.x, v.y, v.z, vel[b].w);
  }
}

// COND launches (the learned solver's extra iterations) use a persistent grid
// and skip the whole launch once the step has converged.
template <bool SCORR, bool LAST, bool COND, int GL>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) kf_dp_update(Dev P, Fast F, int n, size_t stride,
                                                       const int32_t* __restrict__ nbr, const int32_t* __restrict__ cnt,
                                                       const float4* __restrict__ xl, float4* pst,
                                                       const float4* __restrict__ pos, float4* vel,
                                                       const pbf::SolveState* __restrict__ state, float* lamsum) {
  if (COND && state->done) return;
  const int tiles = pbf::tiles_of<GL>(n);
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x)
    dp_update_tile<SCORR, LAST, GL>(tile, P, F, n, stride, nbr, cnt, xl, pst, pos, vel, lamsum);
}

template <bool SCORR, bool LAST, bool COND>
__global__ void __launch_bounds__(kStageThreads) ks_dp_update(Dev P, Fast F, int n, size_t stride,
                                                             const int32_t* __restrict__ nbr,
                                                             const int32_t* __restrict__ cnt,
                                                             const float4* __restrict__ xl, float4* pst,
                                                             const float4* __restrict__ pos, float4* vel,
                                                             const pbf::SolveState* __restrict__ state,
                                                             float* lamsum, TileIO T) {
  __shared__ float4 stage[kStageMax + 1];
  if (COND && state->done) return;
  const int tiles = (n + kTile - 1) / kTile;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int staged = stage_tile<false>(T, tile, xl, stage, nullptr, nullptr);
    if (staged >= 0)
      dp_update_tile<SCORR, LAST, 4, true>(tile, P, F, n, stride, nbr, cnt, xl, pst, pos, vel, lamsum,
                                           Src{T.nbr16, stage, nullptr, staged});
    else
      dp_update_tile<SCORR, LAST, 4>(tile, P, F, n, stride, nbr, cnt, xl, pst, pos, vel, lamsum);
    __syncthreads();
  }
}

// wvis (fast, direct walks): the weights W(r)/rho_q per list entry, written
// by the first pass and read by the final one (pbf::gwalk2w, pbf::gwalkw).
template <bool FINAL, int GL, bool STAGED = false, bool COH = false>
__device__ __forceinline__ void viscosity_tile(int tile, const Fast& F, int n, size_t stride,
                                               const int32_t* __restrict__ nbr, const int32_t* __restrict__ cnt,
                                               const float4* __restrict__ pst, const float4* __restrict__ vin,
                                               float4* vout, float4* posH, float4* pstH,
                                               const uint32_t* __restrict__ origS, uint32_t* origH, __half* wvis,
                                               Src src = Src{nullptr, nullptr, nullptr, 0}) {
  const pbf::Group G = pbf::group_at<GL>(n, tile);
  const int b = G.b;
  const float4 xp = pst[b], vp = vin[b];
  const int c = G.live ? cnt[b] : 0;
  float ax = 0.f, ay = 0.f, az = 0.f;
  auto weight = [&](float4 xq, float4 vq) {
    const float dx = xp.x - xq.x, dy = xp.y - xq.y, dz = xp.z - xq.z;
    const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    return __fdividef(pbf::poly_cube(F, d2), vq.w);
  };
  auto add = [&](float wr, float4 vq) {
    ax = fmaf(vq.x - vp.x, wr, ax);
    ay = fmaf(vq.y - vp.y, wr, ay);
    az = fmaf(vq.z - vp.z, wr, az);
  };
  const int32_t* row = nbr + pbf::list_base(b, stride);
  if (!STAGED && wvis != nullptr) {
    __half* wrow = wvis + pbf::list_base(b, stride);
    if (FINAL)
      pbf::gwalkw<GL, false, COH>(row, wrow, c, n, G.lane, vin, [&](int, float wr, float4 vq) { add(wr, vq); });
    else
      pbf::gwalk2w<GL, COH>(row, wrow, c, n, G.lane, pst, vin, [&](int, float4 xq, float4 vq) {
        const float wr = weight(xq, vq);
        add(wr, vq);
        return wr;
      });
  } else {
    pbf::walk2<GL, STAGED, FINAL, COH>(row, STAGED ? src.nbr16 + (size_t)b * stride : nullptr, c,
                                       STAGED ? src.dummy : n, G.lane, STAGED ? src.a : pst, STAGED ? src.b : vin,
                                       [&](int, float4 xq, float4 vq) { add(weight(xq, vq), vq); });
  }
  ax = pbf::gsum<GL>(ax);
  ay = pbf::gsum<GL>(ay);
  az = pbf::gsum<GL>(az);
  if (!G.live || G.lane != 0) return;
  const float k = F.visc_c * F.visc_poly;
  vout[b] = make_float4(fmaf(k, ax, vp.x), fmaf(k, ay, vp.y), fmaf(k, az, vp.z), vp.w);
  if (FINAL) {
    posH[b] = xp;
    pstH[b] = xp;
    origH[b] = origS[b];
  }
}

template <bool FINAL, int GL>
__global__ void __launch_bounds__(kBlock) kf_viscosity(Dev P, Fast F, int n, size_t stride,
                                                       const int32_t* __restrict__ nbr, const int32_t* __restrict__ cnt,
                                                       const float4* __restrict__ pst, const float4* __restrict__ vin,
                                                       float4* vout, float4* posH, float4* pstH,
                                                       const uint32_t* __restrict__ origS, uint32_t* origH,
                                                       __half* wvis) {
  viscosity_tile<FINAL, GL>(blockIdx.x, F, n, stride, nbr, cnt, pst, vin, vout, posH, pstH, origS, origH, wvis);
}

template <bool FINAL>
__global__ void __launch_bounds__(kStageThreads) ks_viscosity(Dev P, Fast F, int n, size_t stride,
                                                             const int32_t* __restrict__ nbr,
                                                             const int32_t* __restrict__ cnt,
                                                             const float4* __restrict__ pst,
                                                             const float4* __restrict__ vin, float4* vout,
                                                             float4* posH, float4* pstH,
                                                             const uint32_t* __restrict__ origS, uint32_t* origH,
                                                             TileIO T) {
  __shared__ float4 sa[kStageMax + 1], sb[kStageMax + 1];
  const int tile = blockIdx.x;
  const int staged = stage_tile<true>(T, tile, pst, sa, vin, sb);
  if (staged >= 0)
    viscosity_tile<FINAL, 4, true>(tile, F, n, stride, nbr, cnt, pst, vin, vout, posH, pstH, origS, origH, nullptr,
                                   Src{T.nbr16, sa, sb, staged});
  else
    viscosity_tile<FINAL, 4>(tile, F, n, stride, nbr, cnt, pst, vin, vout, posH, pstH, origS, origH, nullptr);
}

template <int GL, bool STAGED = false, bool COH = false>
__device__ __forceinline__ void vorticity_tile(int tile, const Fast& F, int n, size_t stride,
                                               const int32_t* __restrict__ nbr, const int32_t* __restrict__ cnt,
                                               const float4* __restrict__ pst, const float4* __restrict__ vel,
                                               float4* scr, float4* xl, Src src = Src{nullptr, nullptr, nullptr, 0}) {
  const pbf::Group G = pbf::group_at<GL>(n, tile);
  const int b = G.b;
  const float4 xp = pst[b], vp = vel[b];
  const int c = G.live ? cnt[b] : 0;
  float wx = 0.f, wy = 0.f, wz = 0.f;
  pbf::walk2<GL, STAGED, false, COH>(nbr + pbf::list_base(b, stride),
                                     STAGED ? src.nbr16 + (size_t)b * stride : nullptr, c, STAGED ? src.dummy : n,
                                     G.lane, STAGED ? src.a : pst, STAGED ? src.b : vel,
                         [&](int, float4 xq, float4 vq) {
    const float dx = xp.x - xq.x, dy = xp.y - xq.y, dz = xp.z - xq.z;
    const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    const float t = pbf::spikey_over_r(F, d2);
    const float ux = vq.x - vp.x, uy = vq.y - vp.y, uz = vq.z - vp.z;
    // cross(v_q - v_p, del W), del W = spikey * t * r
    wx = fmaf(t, fmaf(uy, dz, -uz * dy), wx);
    wy = fmaf(t, fmaf(uz, dx, -ux * dz), wy);
    wz = fmaf(t, fmaf(ux, dy, -uy * dx), wz);
  });
  wx = pbf::gsum<GL>(wx) * F.spikey;
  wy = pbf::gsum<GL>(wy) * F.spikey;
  wz = pbf::gsum<GL>(wz) * F.spikey;
  if (!G.live || G.lane != 0) return;
  const float wm = sqrtf(fmaf(wz, wz, fmaf(wy, wy, wx * wx)));
  scr[b] = make_float4(wx, wy, wz, wm);
  xl[b] = make_float4(xp.x, xp.y, xp.z, wm);
}

template <int GL>
__global__ void __launch_bounds__(kBlock) kf_vorticity(Dev P, Fast F, int n, size_t stride,
                                                       const int32_t* __restrict__ nbr, const int32_t* __restrict__ cnt,
                                                       const float4* __restrict__ pst, const float4* __restrict__ vel,
                                                       float4* scr, float4* xl) {
  vorticity_tile<GL>(blockIdx.x, F, n, stride, nbr, cnt, pst, vel, scr, xl);
}

__global__ void __launch_bounds__(kStageThreads) ks_vorticity(Dev P, Fast F, int n, size_t stride,
                                                             const int32_t* __restrict__ nbr,
                                                             const int32_t* __restrict__ cnt,
                                                             const float4* __restrict__ pst,
                                                             const float4* __restrict__ vel, float4* scr, float4* xl,
                                                             TileIO T) {
  __shared__ float4 sa[kStageMax + 1], sb[kStageMax + 1];
  const int tile = blockIdx.x;
  const int staged = stage_tile<true>(T, tile, pst, sa, vel, sb);
  if (staged >= 0)
    vorticity_tile<4, true>(tile, F, n, stride, nbr, cnt, pst, vel, scr, xl, Src{T.nbr16, sa, sb, staged});
  else
    vorticity_tile<4>(tile, F, n, stride, nbr, cnt, pst, vel, scr, xl);
}

template <int GL, bool STAGED = false, bool COH = false>
__device__ __forceinline__ void apply_vorticity_tile(int tile, const Fast& F, int n, size_t stride,
                                                     const int32_t* __restrict__ nbr,
                                                     const int32_t* __restrict__ cnt,
                                                     const float4* __restrict__ xl, const float4* __restrict__ scr,
                                                     float4* vel, Src src = Src{nullptr, nullptr, nullptr, 0}) {
  const pbf::Group G = pbf::group_at<GL>(n, tile);
  const int b = G.b;
  const float4 xp = xl[b];
  const int c = G.live ? cnt[b] : 0;
  float ex = 0.f, ey = 0.f, ez = 0.f;
  pbf::walk1<GL, STAGED, false, COH>(nbr + pbf::list_base(b, stride),
                                     STAGED ? src.nbr16 + (size_t)b * stride : nullptr, c, STAGED ? src.dummy : n,
                                     G.lane, STAGED ? src.a : xl, [&](int, float4 xq) {
    const float dx = xp.x - xq.x, dy = xp.y - xq.y, dz = xp.z - xq.z;
    const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    const float t = xq.w * pbf::spikey_over_r(F, d2);
    ex = fmaf(t, dx, ex);
    ey = fmaf(t, dy, ey);
    ez = fmaf(t, dz, ez);
  });
  ex = pbf::gsum<GL>(ex) * F.spikey;
  ey = pbf::gsum<GL>(ey) * F.spikey;
  ez = pbf::gsum<GL>(ez) * F.spikey;
  if (!G.live || G.lane != 0) return;
  const float inv = __fdividef(1.0f, sqrtf(fmaf(ez, ez, fmaf(ey, ey, ex * ex))) + FLT_EPSILON);
  const float Nx = ex * inv, Ny = ey * inv, Nz = ez * inv;
  const float4 wp = scr[b];
  float4 v = vel[b];
  v.x = fmaf(fmaf(Ny, wp.z, -Nz * wp.y), F.vort_dt, v.x);
  v.y = fmaf(fmaf(Nz, wp.x, -Nx * wp.z), F.vort_dt, v.y);
  v.z = fmaf(fmaf(Nx, wp.y, -Ny * wp.x), F.vort_dt, v.z);
  vel[b] = v;
}

template <int GL>
__global__ void __launch_bounds__(kBlock) kf_apply_vorticity(Dev P, Fast F, int n, size_t stride,
                                                             const int32_t* __restrict__ nbr,
                                                             const int32_t* __restrict__ cnt,
                                                             const float4* __restrict__ xl,
                                                             const float4* __restrict__ scr, float4* vel) {
  apply_vorticity_tile<GL>(blockIdx.x, F, n, stride, nbr, cnt, xl, scr, vel);
}

__global__ void __launch_bounds__(kStageThreads) ks_apply_vorticity(Dev P, Fast F, int n, size_t stride,
                                                                   const int32_t* __restrict__ nbr,
                                                                   const int32_t* __restrict__ cnt,
                                                                   const float4* __restrict__ xl,
                                                                   const float4* __restrict__ scr, float4* vel,
                                                                   TileIO T) {
  __shared__ float4 stage[kStageMax + 1];
  const int tile = blockIdx.x;
  const int staged = stage_tile<false>(T, tile, xl, stage, nullptr, nullptr);
  if (staged >= 0)
    apply_vorticity_tile<4, true>(tile, F, n, stride, nbr, cnt, xl, scr, vel, Src{T.nbr16, stage, nullptr, staged});
  else
    apply_vorticity_tile<4>(tile, F, n, stride, nbr, cnt, xl, scr, vel);
}

// ---- the persistent step (batches of scenes) ----
// Every gather pass of a fast-math plain step (K Jacobi iterations of
// density/lambda and delta-p, both XSPH passes, vorticity and its
// application) as ONE launch, after the list fill's.  Work is a queue of tasks, pass-major: task
// (pass, tile) is one tile of that pass, tiles over the batch's sorted slots.
// Blocks take tasks in queue order (an atomic counter) until it is empty.  A
// tile of pass p reads what pass p-1 wrote in the scenes it covers (a list
// never leaves its scene), so it waits only until every tile of pass p-1 that
// covers those scenes has finished: per (pass, scene) counters, each finished
// tile adding one to the counter of every scene it covers.  A scene whose
// pass is done goes on to its next pass while a crowded scene of the batch is
// still in an earlier pass; the launch-per-pass step makes every scene wait
// for the slowest at every pass.
//  - No deadlock: a block waits only on tasks earlier in the queue, which
//    blocks already running have taken; the earliest unfinished task waits on
//    none.  Any grid size works; a persistent one (SMs x resident blocks) is
//    used.
//  - Visibility: a finished tile's writes are fenced (GPU scope) before its
//    counters are raised; a waiting block reads the counters with acquire
//    loads before any of its threads reads the data, and the walks read with
//    plain loads (pbf::ldw<true>), not the read-only path.
//  - Each block fetches its next task while the current one runs, and a
//    block that has found pass p-1 finished in some scenes does not wait for
//    it again for later tiles of pass p in those scenes.
//  - 12 resident blocks per SM (40 registers, a few spilled): measured the
//    fastest of 56, 48 and 40 registers on the 64-scene batch.
//  - Every wait is bounded in time (limit_ns, %globaltimer).  A block that
//    gives up raises PBF_FLAG_WAIT_TIMEOUT and the abort word, and every block
//    then returns at its next task or wait: the launch ends, the step's
//    results are invalid and flagged.
enum PersistKind { kPDensity = 0, kPDp, kPDpLast, kPVisc, kPVort, kPApply, kPViscFinal };
constexpr int kPersistThreads = 128;
constexpr int kPersistTilesPerTask = 1;  // consecutive tiles of one pass per task
constexpr int kPersistMaxK = 16;
constexpr int kPersistMaxPasses = 2 * kPersistMaxK + 4;
// lanes per particle of each gather pass (a tile is kPersistThreads / GL particles)
constexpr int kPGLDensity = 2, kPGLDp = 2, kPGLVisc = 2, kPGLVort = 4, kPGLApply = 2;

struct PersistPass {
  int kind, size, first_task, tiles;  // PersistKind, slots per tile, its first task, its tiles
};
// (tasks of a pass: ceil(tiles / kPersistTilesPerTask))
struct PersistPlan {
  PersistPass pass[kPersistMaxPasses];
  int npass, tasks, nscenes;
  int stall_pass;                // -1, or a pass whose dependency is never met (the wait self-test)
  unsigned long long limit_ns;   // bound of every wait
  uint32_t* words;               // [0] next task, [1] abort
  uint32_t* done;                // [npass][nscenes] finished tiles
  uint32_t* flags;               // PBF_FLAG_WAIT_TIMEOUT is raised here
  const uint32_t* first;         // [nscenes + 1] first slot of every scene, then the slot count
};
struct PersistArrays {
  float4 *pst, *xl, *vel, *velT, *pos, *scr, *velH, *posH, *pstH;
  float* lam;
  __half* wvis;
  uint32_t *nudge, *err, *origH;
  const uint32_t *cell_start, *run_end, *origS;
  int32_t *nbr, *cnt;
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// The last scene whose first slot is <= slot.
__device__ __forceinline__ int persist_scene(const PersistPlan& S, uint32_t slot) {
  int lo = 0, hi = S.nscenes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (S.first[mid] <= slot) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Thread 0 of a block: wait until pass p-1 has finished in scenes sa..sb.
// False when this or another block gave up.
__device__ bool persist_wait(const PersistPlan& S, int p, int sa, int sb) {
  const PersistPass q = S.pass[p - 1];
  const unsigned long long t0 = globaltimer_ns();
  for (int s = sa; s <= sb; ++s) {
    const uint32_t f = S.first[s], e = S.first[s + 1];
    if (e == f) continue;  // an empty scene has no tiles
    uint32_t need = (e - 1) / (uint32_t)q.size - f / (uint32_t)q.size + 1u;
    if (p == S.stall_pass) need += 1u;  // one tile more than exist: the self-test's wait
    const uint32_t* c = S.done + (size_t)(p - 1) * S.nscenes + s;
    unsigned sleep = 128;  // polls back off, so that waiting blocks leave the counters' L2 slice alone
    while (ld_acquire_gpu(c) < need) {
      if (ld_acquire_gpu(S.words + 1) != 0u) return false;
      if (globaltimer_ns() - t0 > S.limit_ns) {
        atomicOr(S.flags, PBF_FLAG_WAIT_TIMEOUT);
        atomicExch(S.words + 1, 1u);
        return false;
      }
      __nanosleep(sleep);
      sleep = min(2u * sleep, 8192u);
    }
  }
  return true;
}

// DRY: the scheduler and its waits only, no tile work (the wait self-test).
template <bool DRY>
__global__ void __launch_bounds__(kPersistThreads, 12)
    k_persist(Dev P, Fast F, int n, size_t stride, PersistPlan S, PersistArrays A) {
  __shared__ int s_task, s_ok;
  // thread 0: the task after the current one (fetched while the current one
  // runs) and the last (pass, scenes) it found finished, which later tasks of
  // the same pass in those scenes need not wait for again
  int next = 0, cp = -1, csa = 0, csb = -1;
  if (threadIdx.x == 0) s_task = (int)atomicAdd(S.words, 1u);
  __syncthreads();
  for (;;) {
    const int task = s_task;
    if (task >= S.tasks) return;
    if (threadIdx.x == 0) next = (int)atomicAdd(S.words, 1u);
    int p = 0;
    while (p + 1 < S.npass && task >= S.pass[p + 1].first_task) ++p;
    const int kind = S.pass[p].kind, size = S.pass[p].size;
    const int t0 = (task - S.pass[p].first_task) * kPersistTilesPerTask;
    const int t1 = min(t0 + kPersistTilesPerTask, S.pass[p].tiles);
    const uint32_t a = (uint32_t)t0 * (uint32_t)size;
    const uint32_t z = min((uint32_t)t1 * (uint32_t)size, (uint32_t)n) - 1u;
    const int sa = persist_scene(S, a), sb = persist_scene(S, z);
    if (threadIdx.x == 0) {
      bool ok = true;
      if (p > 0 && !(p == cp && sa >= csa && sb <= csb)) {
        ok = persist_wait(S, p, sa, sb);
        __threadfence();
        cp = p;
        csa = sa;
        csb = sb;
      }
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) return;
    for (int tile = t0; !DRY && tile < t1; ++tile) {
      switch (kind) {
        case kPDensity: {
          float err = 0.0f;
          const LearnIO io{};
          density_lambda_tile<kDlPlain, kPGLDensity, false, true>(tile, P, F, n, stride, A.nbr, A.cnt, A.pst, A.xl,
                                                                  A.vel, A.lam, A.nudge, io, err);
          break;
        }
        case kPDp:
          dp_update_tile<false, false, kPGLDp, false, true>(tile, P, F, n, stride, A.nbr, A.cnt, A.xl, A.pst, A.pos,
                                                            A.vel, nullptr);
          break;
        case kPDpLast:
          dp_update_tile<false, true, kPGLDp, false, true>(tile, P, F, n, stride, A.nbr, A.cnt, A.xl, A.pst, A.pos,
                                                           A.vel, nullptr);
          break;
        case kPVisc:
          viscosity_tile<false, kPGLVisc, false, true>(tile, F, n, stride, A.nbr, A.cnt, A.pst, A.vel, A.velT,
                                                       nullptr, nullptr, nullptr, nullptr, A.wvis);
          break;
        case kPVort:
          vorticity_tile<kPGLVort, false, true>(tile, F, n, stride, A.nbr, A.cnt, A.pst, A.velT, A.scr, A.xl);
          break;
        case kPApply:
          apply_vorticity_tile<kPGLApply, false, true>(tile, F, n, stride, A.nbr, A.cnt, A.xl, A.scr, A.velT);
          break;
        default:
          viscosity_tile<true, kPGLVisc, false, true>(tile, F, n, stride, A.nbr, A.cnt, A.pst, A.velT, A.velH,
                                                      A.posH, A.pstH, A.origS, A.origH, A.wvis);
          break;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();  // the tiles' writes before their counters
      for (int tile = t0; tile < t1; ++tile) {
        const uint32_t ta = (uint32_t)tile * (uint32_t)size;
        const uint32_t tz = min(ta + (uint32_t)size, (uint32_t)n) - 1u;
        const int ua = persist_scene(S, ta), ub = persist_scene(S, tz);
        for (int s = ua; s <= ub; ++s) atomicAdd(S.done + (size_t)p * S.nscenes + s, 1u);
      }
      s_task = *(volatile const uint32_t*)(S.words + 1) ? S.tasks : next;  // another block gave up: stop
    }
    __syncthreads();
  }
}

// Residual statistics (no state change): density over the current lists,
// clamped error, kinetic energy, centre of mass, list lengths.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kBlock) k_stats(Dev P, int b0, int b1, size_t stride,
                                                  const int32_t* __restrict__ nbr,
                                                  const int32_t* __restrict__ cnt, const float4* __restrict__ pst,
                                                  const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                  double* acc, unsigned long long* maxerr,
                                                  unsigned long long* hits) {
  const int b = b0 + blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0, ke = 0.0, cx = 0.0, cy = 0.0, cz = 0.0, nn = 0.0;
  if (b < b1) {
    const float4 xp = pst[b];
    const int c = cnt[b];
    float d = pbf::xmul(P.m, P.W0);
    for (int k = 0; k < c; ++k) {
      const float4 xq = pst[nbr[pbf::list_at(b, stride, k)]];
      const float rx = pbf::xsub(xp.x, xq.x), ry = pbf::xsub(xp.y, xq.y), rz = pbf::xsub(xp.z, xq.z);
      d = pbf::xadd(d, pbf::xmul(P.m, pbf::poly6<true>(P, __fsqrt_rn(pbf::mag2<true>(rx, ry, rz)))));
    }
    e = (double)d / (double)P.rho0 - 1.0;
    if (e < 0.0) e = 0.0;
    atomicMax(maxerr, (unsigned long long)__double_as_longlong(e));
    const float4 v = vel[b];
    ke = 0.5 * (double)P.m * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
    const float4 x = pos[b];
    cx = x.x; cy = x.y; cz = x.z;
    nn = c;
    if (c >= P.cap) atomicAdd(hits, 1ull);
  }
  e = warp_sum(e); ke = warp_sum(ke); cx = warp_sum(cx); cy = warp_sum(cy); cz = warp_sum(cz); nn = warp_sum(nn);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&acc[0], e); atomicAdd(&acc[1], ke); atomicAdd(&acc[2], cx);
    atomicAdd(&acc[3], cy); atomicAdd(&acc[4], cz); atomicAdd(&acc[5], nn);
  }
}

// Neighbour lists in reference index space, [N][cap], -1 past count.
// seg (fast math, whose last fill walked in slot order when *last_order is
// 1): each slot-order list is written back in the reference's order, visit
// by visit (x offset outer, z inner; within a visit the entries keep their
// ascending slots), from where the fill recorded each visit starts.
__global__ void k_export_neighbors(int n, size_t stride, int cap, const int32_t* __restrict__ nbr,
                                   const int32_t* __restrict__ cnt, const uint32_t* __restrict__ orig,
                                   int32_t* idx_out, int32_t* cnt_out, const uint32_t* __restrict__ seg,
                                   const uint32_t* __restrict__ last_order) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const size_t o = orig[b];
  const int c = cnt[b];
  if (cnt_out) cnt_out[o] = c;
  if (!idx_out) return;
  const uint8_t* sc = seg && *last_order ? reinterpret_cast<const uint8_t*>(seg + (size_t)b * kSegWords) : nullptr;
  if (sc == nullptr || sc[27] == kSegReferenceOrder) {
    for (int k = 0; k < cap; ++k)
      idx_out[o * cap + k] = k < c ? (int32_t)orig[nbr[pbf::list_at(b, stride, k)]] : -1;
    return;
  }
  int e = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) {
        const int v = k * 9 + j * 3 + i;  // visit v's entries: [sc[v], sc[v+1]) of the slot-order list
        for (int t = sc[v], t1 = v < 26 ? sc[v + 1] : c; t < t1; ++t)
          idx_out[o * cap + e++] = (int32_t)orig[nbr[pbf::list_at(b, stride, t)]];
      }
  for (; e < cap; ++e) idx_out[o * cap + e] = -1;
}

}  // namespace

// ============================================================================
// Context
// ============================================================================
struct pbf_ctx {
  pbf_params params{};
  Dev dev{};
  Fast fast{};
  size_t capacity = 0, n = 0;
  int64_t dims[3] = {0, 0, 0};
  int nbins = 0, nscan_parts = 0;
  int nbins_cap = 0;   // bins the cell arrays were allocated for
  size_t lstride = 0;      // list row stride: neighbor_cap rounded up to kListAlign entries
  size_t lstride_cap = 0;  // list row stride the list buffer was allocated for
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;  // captures the body of the learned solver's conditional loop
  bool capture_failed = false;  // a step's conditional loop could not be captured whole
  bool lists_valid = false;
  bool lists_slot_order = false;  // fast math: seg says, per list, which order it is in
  uint32_t* fill_words = nullptr;  // [kFillWords] the fast fill's order choice (FillWord)
  int32_t* redo_queue = nullptr;   // [C] slot-order lists that reached the cap
  uint32_t* seg = nullptr;        // [C][kSegWords] where the fast fill's visits start

  float4 *posH = nullptr, *pstH = nullptr, *velH = nullptr, *scrH = nullptr;
  float4 *posS = nullptr, *pstS = nullptr, *velS = nullptr, *scrS = nullptr, *xl = nullptr, *velT = nullptr;
  float *lamH = nullptr, *lamS = nullptr;
  uint32_t *origH = nullptr, *origS = nullptr, *key = nullptr, *keyH = nullptr;
  uint32_t* run_end = nullptr;  // per sorted slot: end of its run of bit-identical x* (k_runs)
  // radix sort: keys at the reference index and their ping-pong twin, digit
  // histograms, their scan, scan partials; `sorted` = the pair buffer holding
  // the sorted pairs after the last pass
  uint32_t *key_ref = nullptr, *key_alt = nullptr, *radix_hist = nullptr, *radix_off = nullptr,
           *radix_parts = nullptr;
  int radix_passes = 0;
  unsigned long long* sorted = nullptr;
  uint32_t *cell_count = nullptr, *cell_start = nullptr, *scan_part = nullptr, *err = nullptr, *nudge = nullptr;
  unsigned long long *pairs = nullptr, *pairs_sorted = nullptr;
  int32_t *nbr = nullptr, *cnt = nullptr;
  __half* wvis = nullptr;  // XSPH weights per list entry (the list's layout, half precision), in stage_i's memory
  float* stage = nullptr;  // 6*C floats: two AoS float3 staging areas
  // neighbor export staging (C*cap + C); within a step, the XSPH weights
  // (wvis: written by the first viscosity pass, read by the final one)
  int32_t* stage_i = nullptr;
  double* acc = nullptr;
  unsigned long long *maxerr = nullptr, *hits = nullptr;

  // learned warm start
  float *lamsumH = nullptr, *lamprevS = nullptr, *feats = nullptr;
  __nv_bfloat16* featb = nullptr;  // [C][16] normalised features of the warm iteration
  pbf::SolveState* state = nullptr;
  double* partials = nullptr;  // [partials_cap] residual check sums, one per block
  bool recording = false;
  float *mlp_params = nullptr, *mlp_grad = nullptr, *mlp_m = nullptr, *mlp_v = nullptr, *mlp_norm = nullptr;
  float* mlp_loss = nullptr;
  __nv_bfloat16 *w1b = nullptr, *w2b = nullptr, *w2tb = nullptr;
  float label_scale = 1.0f;
  int adam_t = 0;
  bool mlp_ready = false;
  uint64_t steps_done = 0;  // steps advanced by pbf_step (saved with the state)
  // launch shapes of the fast gather families, and the persistent grids of
  // the learned solver's skippable launches (SMs x resident blocks)
  pbf_tuning tune{{2, 2, 2, 4, 2}, {128, 128, kBlock, kBlock, kBlock}, {0, 0, 0, 0, 0}};  // pbf.h's defaults
  int sms = 148;
  int pgrid_check = 148, pgrid_dp = 148;
  // staged gathers: tile descriptors and the 16-bit lists the list fill writes
  int32_t *tile_nruns = nullptr, *tile_total = nullptr;
  int4* tile_runs = nullptr;
  uint16_t* nbr16 = nullptr;
  int partials_cap = 0;

  // batch of scenes (empty: one scene, the parameter block's box); the device
  // copies back Dev::scenes and Dev::scene_first
  std::vector<pbf_scene> scenes;
  std::vector<pbf::Region> regions;
  std::vector<uint32_t> scene_first;
  pbf::Region* d_regions = nullptr;
  uint32_t* d_scene_first = nullptr;

  // persistent step (pbf_set_persistent): its task counter and abort word,
  // the [pass][scene] tile counters, the grid
  bool persistent = false;
  uint32_t *persist_words = nullptr, *persist_done = nullptr;
  int persist_grid = 0;

  std::map<int, cudaGraphExec_t> graphs;
  uint64_t graph_epoch = 0;  // counts drop_graphs: a scene group rebuilds when a member's changes
  std::vector<void*> allocations;

  bool timing = false;
  struct Mark {
    const char* name;
    cudaEvent_t start, stop;
  };
  std::vector<Mark> marks;
  size_t marks_used = 0;
  std::map<std::string, std::pair<int64_t, double>> times;
  std::vector<std::string> time_order;

  std::string error;
};

namespace {

thread_local std::string g_create_error;

int fail(pbf_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->error = buf; else g_create_error = buf;
  return code;
}

#define CK(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(ctx, PBF_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));        \
  } while (0)

int check_launch(pbf_ctx* ctx, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ctx, PBF_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return PBF_OK;
}

// Build the device constant block from the public parameters (all derived
// constants are evaluated on the host in the reference's types).
int make_dev(pbf_ctx* ctx, const pbf_params& p, Dev& d, int64_t dims[3]) {
  if (!(p.time_step > 0.0f) || !(p.smoothing_radius > 0.0f) || !(p.neighbor_bin_spacing > 0.0f) ||
      !(p.rest_density > 0.0f) || !(p.rest_mass > 0.0f))
    return fail(ctx, PBF_ERR_PARAMS, "time_step, smoothing_radius, neighbor_bin_spacing, rest_density and "
                                     "rest_mass must be > 0");
  if (p.solve_steps < 0) return fail(ctx, PBF_ERR_PARAMS, "solve_steps must be >= 0");
  if (p.solver != 0 && p.solver != 1) return fail(ctx, PBF_ERR_PARAMS, "solver must be 0 (plain) or 1 (learned)");
  if (p.solver == 1 && p.exact_math)
    return fail(ctx, PBF_ERR_PARAMS, "the learned warm start runs in fast math only (exact_math = 0)");
  if (p.solver == 1 && (p.max_iterations < 1 || p.max_iterations > 64))
    return fail(ctx, PBF_ERR_PARAMS, "max_iterations must be in [1, 64]");
  if (p.neighbor_cap < 1 || p.neighbor_cap > 64)
    return fail(ctx, PBF_ERR_PARAMS, "neighbor_cap must be in [1, 64], got %d", p.neighbor_cap);
  const float s = p.neighbor_bin_spacing;
  for (int a = 0; a < 3; ++a) {
    if (!(p.boundary_max[a] > p.boundary_min[a]))
      return fail(ctx, PBF_ERR_PARAMS, "boundary max must exceed min on every axis");
    // The reference's bin hash casts floor((x+s)/s) to size_t, defined only
    // for x >= -s; every clamped position and its +-s re-hash must land in
    // the grid (neighbors.h:69-71, 109-114, 172-185).
    if (p.boundary_min[a] < 0.0f)
      return fail(ctx, PBF_ERR_PARAMS, "boundary min must be >= 0 (reference bin hash, neighbors.h:109-114)");
    dims[a] = pbf::grid_dim(p.boundary_max[a] - p.boundary_min[a], s);
    const float lo = (p.boundary_min[a] - s);
    const float hi = (p.boundary_max[a] + s);
    if (pbf::axis_bin(lo, s) < 0 || pbf::axis_bin(hi, s) > dims[a] - 1)
      return fail(ctx, PBF_ERR_PARAMS,
                  "axis %d: the reference grid (ceil(extent/s)+2 = %lld bins) does not cover the boundary "
                  "and its +-s neighbour bins; a box with min 0 and max not a multiple of s does",
                  a, (long long)dims[a]);
  }
  const double nb = (double)dims[0] * (double)dims[1] * (double)dims[2];
  if (nb >= 2147483647.0) return fail(ctx, PBF_ERR_PARAMS, "grid of %.0f bins exceeds 2^31", nb);
  std::memset(&d, 0, sizeof(d));
  d.span_end = 0xffffffffu;
  const float h = p.smoothing_radius;
  d.dt = p.time_step;
  d.gdt = p.gravity * p.time_step;
  d.h = h;
  d.s = s;
  d.s2 = s * s;
  d.m = p.rest_mass;
  d.rho0 = p.rest_density;
  d.inv_rho0 = 1.0f / p.rest_density;
  d.neg_inv_rho0 = -1.0f / p.rest_density;
  d.poly6_norm = (float)(315.0 / (64.0 * M_PI * std::pow((double)h, 9.0)));
  d.spikey_norm = (float)(-45.0 / (M_PI * std::pow((double)h, 6.0)));
  d.cspline_norm = (float)(32.0 / (M_PI * std::pow((double)h, 9.0)));
  {
    const float a = h * h - 0.0f * 0.0f;
    d.W0 = d.poly6_norm * a * a * a;
  }
  d.lambda_eps = p.lambda_epsilon;
  d.visc_c = p.visc_c;
  d.vort_eps = p.vorticity_coef;
  d.gamma = p.gamma;
  for (int a = 0; a < 3; ++a) {
    d.bmin[a] = p.boundary_min[a];
    d.bmax[a] = p.boundary_max[a];
    d.mc[a] = p.mover_center[a];
  }
  d.mr = p.mover_radius;
  d.mr2 = p.mover_radius * p.mover_radius;
  d.scorr_k = p.scorr_k;
  d.scorr_n = p.scorr_n;
  if (p.scorr_k > 0.0f) {
    const float r = p.scorr_dq * h;
    float w = 0.0f;
    if (!(r > h)) {
      const float a = h * h - r * r;
      w = d.poly6_norm * a * a * a;
    }
    if (!(w > 0.0f)) return fail(ctx, PBF_ERR_PARAMS, "scorr_dq must be in (0, 1)");
    d.inv_wdq = 1.0f / w;
  }
  d.vthr = 0.000001 * (double)p.max_speed;
  d.h_eps = (double)h * 0.000001;
  {
    // margin of the bin-skip test in k_fill2: 64 ulps of the largest hashed coordinate
    float mx = 0.0f;
    for (int a = 0; a < 3; ++a) mx = std::fmax(mx, std::fabs(p.boundary_max[a]) + 2.0f * s);
    d.skip_eps = 64.0f * std::ldexp(1.0f, std::ilogb(mx) - 23);
  }
  d.dimx = (int)dims[0];
  d.dimy = (int)dims[1];
  d.dimz = (int)dims[2];
  d.nbins = (int)(dims[0] * dims[1] * dims[2]);
  d.cap = p.neighbor_cap;
  return PBF_OK;
}

// Dev of a batch: every scene validated as a single scene with its own box;
// the physics of scene 0 (the same for all: only the box differs), the total
// bin count, the widest bin-skip margin, and the host tables of regions and
// first slots.
int make_dev_batch(pbf_ctx* ctx, const pbf_params& p, const std::vector<pbf_scene>& sc, Dev& d,
                   std::vector<pbf::Region>& regions, std::vector<uint32_t>& first) {
  regions.clear();
  first.clear();
  int64_t total = 0;
  size_t slot = 0;
  float skip = 0.0f;
  for (size_t i = 0; i < sc.size(); ++i) {
    pbf_params q = p;
    for (int a = 0; a < 3; ++a) {
      q.boundary_min[a] = sc[i].boundary_min[a];
      q.boundary_max[a] = sc[i].boundary_max[a];
    }
    Dev di;
    int64_t dims[3];
    if (int rc = make_dev(ctx, q, di, dims)) {
      const std::string why = ctx->error;
      return fail(ctx, rc, "scene %zu: %s", i, why.c_str());
    }
    if (i == 0) d = di;
    pbf::Region r;
    for (int a = 0; a < 3; ++a) {
      r.bmin[a] = q.boundary_min[a];
      r.bmax[a] = q.boundary_max[a];
    }
    r.dimx = di.dimx;
    r.dimy = di.dimy;
    r.dimz = di.dimz;
    r.key0 = (uint32_t)total;
    regions.push_back(r);
    first.push_back((uint32_t)slot);
    total += di.nbins;
    slot += sc[i].count;
    skip = std::max(skip, di.skip_eps);
    if (total >= 2147483647ll) return fail(ctx, PBF_ERR_PARAMS, "the batch's grids exceed 2^31 bins");
  }
  first.push_back((uint32_t)slot);
  d.nbins = (int)total;
  d.skip_eps = skip;
  d.nscenes = (int)sc.size();
  return PBF_OK;
}

// Copy the batch's tables to the device and point Dev at them.
int upload_scenes(pbf_ctx* ctx) {
  if (ctx->scenes.empty()) return PBF_OK;
  CK(cudaMemcpy(ctx->d_regions, ctx->regions.data(), ctx->regions.size() * sizeof(pbf::Region),
                cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_scene_first, ctx->scene_first.data(), ctx->scene_first.size() * sizeof(uint32_t),
                cudaMemcpyHostToDevice));
  ctx->dev.scenes = ctx->d_regions;
  ctx->dev.scene_first = ctx->d_scene_first;
  ctx->dev.nscenes = (int)ctx->scenes.size();
  return PBF_OK;
}

template <typename T>
int dalloc(pbf_ctx* ctx, T** ptr, size_t count) {
  void* p = nullptr;
  const size_t bytes = count * sizeof(T) > 0 ? count * sizeof(T) : 16;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess)
    return fail(ctx, PBF_ERR_CUDA, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
  ctx->allocations.push_back(p);
  *ptr = static_cast<T*>(p);
  return PBF_OK;
}

void drop_graphs(pbf_ctx* ctx) {
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
  ctx->graph_epoch++;
}

// The configurations the persistent step runs: a batch of scenes, fast math,
// the plain solver with 1..kPersistMaxK iterations, no surface tension, no
// s_corr.  Any other runs the launch-per-pass step.
bool persist_supported(const pbf_ctx* ctx) {
  const pbf_params& p = ctx->params;
  return !ctx->scenes.empty() && !p.exact_math && p.solver == 0 && p.gamma == 0.0f && !(p.scorr_k > 0.0f) &&
         p.solve_steps >= 1 && p.solve_steps <= kPersistMaxK;
}
bool persist_on(const pbf_ctx* ctx) { return ctx->persistent && persist_supported(ctx) && ctx->n > 0; }

// The task queue of one persistent step over the context's n slots.
PersistPlan persist_plan(const pbf_ctx* ctx) {
  PersistPlan S{};
  const int n = (int)ctx->n;
  int np = 0, task = 0;
  auto add = [&](int kind, int size) {
    const int tiles = (n + size - 1) / size;
    S.pass[np++] = PersistPass{kind, size, task, tiles};
    task += (tiles + kPersistTilesPerTask - 1) / kPersistTilesPerTask;
  };
  const int K = ctx->params.solve_steps;
  for (int it = 0; it < K; ++it) {
    add(kPDensity, kPersistThreads / kPGLDensity);
    add(it == K - 1 ? kPDpLast : kPDp, kPersistThreads / kPGLDp);
  }
  add(kPVisc, kPersistThreads / kPGLVisc);
  add(kPVort, kPersistThreads / kPGLVort);
  add(kPApply, kPersistThreads / kPGLApply);
  add(kPViscFinal, kPersistThreads / kPGLVisc);
  S.npass = np;
  S.tasks = task;
  S.nscenes = (int)ctx->scenes.size();
  S.stall_pass = -1;
  S.limit_ns = 2000000000ull;  // 2 s: far above any tile's work, short of a watchdog
  S.words = ctx->persist_words;
  S.done = ctx->persist_done;
  S.flags = ctx->err;
  S.first = ctx->d_scene_first;
  return S;
}


// Stage spans are [0, e) with e <= n: the particles of reference index below
// e (a multi-rank driver's resident particles, Simulation/Source/main.adios);
// the others are halo particles the stage reads but leaves as they are.
int check_span(pbf_ctx* ctx, size_t b, size_t e) {
  if (b != 0 || e > ctx->n)
    return fail(ctx, PBF_ERR_SPAN, "span [%zu, %zu) given; spans are [0, e) with e <= %zu particles", b, e,
                ctx->n);
  return PBF_OK;
}

// The constant block of a per-stage call over the span [0, e).
Dev span_dev(const pbf_ctx* ctx, size_t e) {
  Dev d = ctx->dev;
  if (e < ctx->n) {
    d.span_orig = ctx->origH;
    d.span_end = (uint32_t)e;
  }
  return d;
}

int need_lists(pbf_ctx* ctx) {
  if (!ctx->lists_valid) return fail(ctx, PBF_ERR_STATE, "no neighbor lists: call find_neighbors first");
  return PBF_OK;
}

// ---- launch shapes of the fast gather kernels ----
// fn(std::integral_constant<int, GL>) for the lanes-per-particle of a shape.
template <class Fn>
void with_lanes(int lanes, Fn&& fn) {
  if (lanes == 4)
    fn(std::integral_constant<int, 4>{});
  else if (lanes == 2)
    fn(std::integral_constant<int, 2>{});
  else
    fn(std::integral_constant<int, 8>{});
}

bool shape_ok(int lanes, int block, int staged) {
  if (staged) return staged == 1 && lanes == 4 && block == kStageThreads;
  return (lanes == 2 || lanes == 4 || lanes == 8) && (block == 128 || block == 256);
}

bool any_staged(const pbf_ctx* ctx) {
  if (ctx->params.exact_math) return false;
  for (int f = 0; f < PBF_TUNE_FAMILIES; ++f)
    if (ctx->tune.staged[f]) return true;
  return false;
}

TileIO tile_io(const pbf_ctx* ctx) { return TileIO{ctx->tile_nruns, ctx->tile_total, ctx->tile_runs, ctx->nbr16}; }


// The tensor-core network: a persistent grid of at most 6 CTAs per SM (the
// most that 33 KB of shared memory each lets reside; 6 x 64 of the SM's 512
// TMEM columns), never more CTAs than tiles.
int mlp_tc_grid(const pbf_ctx* ctx, int n) {
  const int tiles = (n + pbf::tc::kRows - 1) / pbf::tc::kRows;
  return std::max(1, std::min(tiles, 6 * ctx->sms));
}

int grid_of(const pbf_ctx* ctx, int family) {
  if (ctx->tune.staged[family]) return (int)((ctx->n + kTile - 1) / kTile);
  return blocks_for(ctx->n * (size_t)ctx->tune.lanes[family], ctx->tune.block[family]);
}

// Persistent grids of the residual check and the conditional delta-p pass for
// the current shapes: SMs x resident blocks, at most partials_cap.
int update_shapes(pbf_ctx* ctx) {
  auto resident = [&](const void* fn, int block) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, 0) != cudaSuccess || per_sm <= 0)
      per_sm = 1;
    return std::min(ctx->sms * per_sm, ctx->partials_cap);
  };
  const pbf_tuning& t = ctx->tune;
  if (t.staged[PBF_TUNE_DENSITY])
    ctx->pgrid_check = std::min(resident((const void*)ks_density_lambda<kDlCheck, false>, kStageThreads),
                                resident((const void*)ks_density_lambda<kDlCheck, true>, kStageThreads));
  else
    with_lanes(t.lanes[PBF_TUNE_DENSITY], [&](auto gl) {
      constexpr int GL = decltype(gl)::value;
      ctx->pgrid_check = std::min(resident((const void*)kf_density_lambda<kDlCheck, GL, false>, t.block[PBF_TUNE_DENSITY]),
                                  resident((const void*)kf_density_lambda<kDlCheck, GL, true>, t.block[PBF_TUNE_DENSITY]));
    });
  if (t.staged[PBF_TUNE_DELTA_P])
    ctx->pgrid_dp = resident((const void*)ks_dp_update<false, false, true>, kStageThreads);
  else
    with_lanes(t.lanes[PBF_TUNE_DELTA_P], [&](auto gl) {
      ctx->pgrid_dp = resident((const void*)kf_dp_update<false, false, true, decltype(gl)::value>,
                               t.block[PBF_TUNE_DELTA_P]);
    });
  cudaGetLastError();  // occupancy queries leave no error behind
  return PBF_OK;
}

// ---- launch bookkeeping: per-kernel CUDA events when timing is on ----
struct Launch {
  pbf_ctx* ctx;
  const char* name;
  explicit Launch(pbf_ctx* c, const char* nm) : ctx(c), name(nm) {
    if (!ctx->timing) return;
    if (ctx->marks_used == ctx->marks.size()) {
      pbf_ctx::Mark m{nm, nullptr, nullptr};
      cudaEventCreate(&m.start);
      cudaEventCreate(&m.stop);
      ctx->marks.push_back(m);
    }
    ctx->marks[ctx->marks_used].name = nm;
    cudaEventRecord(ctx->marks[ctx->marks_used].start, ctx->stream);
  }
  ~Launch() {
    if (!ctx->timing) return;
    cudaEventRecord(ctx->marks[ctx->marks_used].stop, ctx->stream);
    ctx->marks_used++;
  }
};

int harvest_times(pbf_ctx* ctx) {
  if (!ctx->timing || ctx->marks_used == 0) return PBF_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  for (size_t i = 0; i < ctx->marks_used; ++i) {
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, ctx->marks[i].start, ctx->marks[i].stop));
    auto it = ctx->times.find(ctx->marks[i].name);
    if (it == ctx->times.end()) {
      ctx->times[ctx->marks[i].name] = {1, (double)ms};
      ctx->time_order.push_back(ctx->marks[i].name);
    } else {
      it->second.first += 1;
      it->second.second += ms;
    }
  }
  ctx->marks_used = 0;
  return PBF_OK;
}

// ---- neighbor build ----
// Hash + histogram must already have produced key/rank/cell_count.
void launch_sort_to_pairs(pbf_ctx* ctx) {
  const int n = (int)ctx->n;
  const int m = ctx->nbins;  // scan m entries -> m+1 outputs
  cudaStream_t s = ctx->stream;
  {
    Launch L(ctx, "scan_reduce");
    k_scan_reduce<<<ctx->nscan_parts, kScanThreads, 0, s>>>(ctx->cell_count, m, ctx->scan_part);
  }
  {
    Launch L(ctx, "scan_partials");
    k_scan_partials<<<1, kScanThreads, 0, s>>>(ctx->scan_part, ctx->nscan_parts);
  }
  {
    Launch L(ctx, "scan_apply");
    k_scan_apply<<<ctx->nscan_parts, kScanThreads, 0, s>>>(ctx->cell_count, m, ctx->scan_part, ctx->cell_start);
  }
  // stable LSD radix sort of (key, pair), input in reference-index order
  const int tiles = (int)(((size_t)n + kRadixTile - 1) / kRadixTile);
  const int hm = kRadixDigits * tiles;
  const int hp = (int)(((size_t)hm + 1 + kScanTile - 1) / kScanTile);
  uint32_t* kin = ctx->key_ref;
  uint32_t* kout = ctx->key_alt;
  unsigned long long* vin = ctx->pairs;
  unsigned long long* vout = ctx->pairs_sorted;
  for (int p = 0; p < ctx->radix_passes; ++p) {
    const int shift = p * kRadixBits;
    const bool last = p == ctx->radix_passes - 1;
    {
      Launch L(ctx, "radix_hist");
      k_radix_hist<<<tiles, kRadixThreads, 0, s>>>(kin, n, shift, tiles, ctx->radix_hist);
    }
    {
      Launch L(ctx, "radix_scan");
      k_scan_reduce<<<hp, kScanThreads, 0, s>>>(ctx->radix_hist, hm, ctx->radix_parts);
    }
    {
      Launch L(ctx, "radix_scan");
      k_scan_partials<<<1, kScanThreads, 0, s>>>(ctx->radix_parts, hp);
    }
    {
      Launch L(ctx, "radix_scan");
      k_scan_apply<<<hp, kScanThreads, 0, s>>>(ctx->radix_hist, hm, ctx->radix_parts, ctx->radix_off);
    }
    {
      Launch L(ctx, "radix_scatter");
      k_radix_scatter<<<tiles, kRadixThreads, 0, s>>>(kin, vin, n, shift, tiles, ctx->radix_off,
                                                     last ? nullptr : kout, vout);
    }
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  ctx->sorted = vin;  // the last pass's output (the input itself when no pass is needed)
}

void launch_fill(pbf_ctx* ctx, const float4* pst) {
  {
    Launch L(ctx, "runs");
    k_runs<<<blocks_for(ctx->n, kRunBlock), kRunBlock, 0, ctx->stream>>>((int)ctx->n, pst, ctx->run_end,
                                                                         ctx->cell_count + ctx->nbins);
  }
  // fast math: lists in slot order while few reach the cap (the gathers' sums
  // in any order are within the fast path's tolerance), the capped ones
  // walked again in the reference's order; exact math: the reference's order
  const bool slot = ctx->params.exact_math == 0;
  ctx->lists_slot_order = slot;
  {
    Launch L(ctx, "fill_neighbors");
    auto fill = [&](auto stage, auto order) {
      k_fill2<decltype(stage)::value, decltype(order)::value>
          <<<blocks_for(ctx->n, kFillBlock), kFillBlock, 0, ctx->stream>>>(
              ctx->dev, (int)ctx->n, ctx->lstride, pst, ctx->cell_start, ctx->run_end, ctx->nbr, ctx->cnt, ctx->err,
              tile_io(ctx), ctx->seg, ctx->fill_words, ctx->redo_queue);
    };
    using T_ = std::true_type;
    using F_ = std::false_type;
    if (any_staged(ctx)) {
      if (slot) fill(T_{}, T_{}); else fill(T_{}, F_{});
    } else {
      if (slot) fill(F_{}, T_{}); else fill(F_{}, F_{});
    }
  }
  if (slot) {
    Launch L(ctx, "fill_redo");
    const int grid = std::max(1, std::min(blocks_for(ctx->n, kFillBlock), 4 * ctx->sms));
    k_fill_redo<<<grid, kFillBlock, 0, ctx->stream>>>(ctx->dev, (int)ctx->n, ctx->lstride, pst, ctx->cell_start,
                                                      ctx->run_end, ctx->nbr, ctx->cnt, ctx->err, ctx->redo_queue,
                                                      ctx->fill_words);
  }
}

// An upload starts the fast fill's order choice afresh: slot order first, no
// lists counted.  The steps from an uploaded state then do not depend on what
// the context ran before.
int reset_fill_order(pbf_ctx* ctx) {
  CK(cudaMemsetAsync(ctx->fill_words, 0, kFillWords * sizeof(uint32_t), ctx->stream));
  CK(cudaMemsetAsync(ctx->fill_words + kFillSlotOrder, 1, 1, ctx->stream));
  return PBF_OK;
}

// The list fill, then every gather pass of the step in one launch.
void launch_persistent(pbf_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  const int n = (int)ctx->n;
  launch_fill(ctx, ctx->pstS);
  const PersistPlan S = persist_plan(ctx);
  cudaMemsetAsync(ctx->persist_words, 0, 2 * sizeof(uint32_t), s);
  cudaMemsetAsync(ctx->persist_done, 0, (size_t)S.npass * S.nscenes * sizeof(uint32_t), s);
  PersistArrays A{};
  A.pst = ctx->pstS;
  A.xl = ctx->xl;
  A.vel = ctx->velS;
  A.velT = ctx->velT;
  A.pos = ctx->posS;
  A.scr = ctx->scrH;
  A.velH = ctx->velH;
  A.posH = ctx->posH;
  A.pstH = ctx->pstH;
  A.lam = ctx->lamH;
  A.wvis = ctx->wvis;
  A.nudge = ctx->nudge;
  A.err = ctx->err;
  A.origH = ctx->origH;
  A.cell_start = ctx->cell_start;
  A.run_end = ctx->run_end;
  A.origS = ctx->origS;
  A.nbr = ctx->nbr;
  A.cnt = ctx->cnt;
  Launch L(ctx, "persistent_step");
  k_persist<false><<<ctx->persist_grid, kPersistThreads, 0, s>>>(ctx->dev, ctx->fast, n, ctx->lstride, S, A);
}

// ---- the fused step (graph-capturable: fixed pointers, no host sync) ----
pbf::MlpDev mlp_dev(const pbf_ctx* ctx) {
  pbf::MlpDev M;
  M.w1 = ctx->w1b;
  M.w2 = ctx->w2b;
  M.w2t = ctx->w2tb;
  M.b1 = ctx->mlp_params + pbf::kOffB1;
  M.b2 = ctx->mlp_params + pbf::kOffB2;
  M.w3 = ctx->mlp_params + pbf::kOffW3;
  M.b3 = ctx->mlp_params + pbf::kOffB3;
  M.feat_mean = ctx->mlp_norm;
  M.feat_inv_std = ctx->mlp_norm + pbf::kMlpIn;
  M.label_scale = ctx->label_scale;
  return M;
}

// The learned warm start's Jacobi loop: iteration 1 with the MLP's lambda,
// then up to max_iterations-1 plain iterations, each run only while the mean
// clamped density error at the current x* exceeds residual_tol (a check pass
// decides; once converged, the remaining launches return at once), a final
// check recording the step's residual, and the velocity update.
template <bool SCORR>
void launch_learned_solve(pbf_ctx* ctx) {
  const int n = (int)ctx->n;
  const size_t st = ctx->lstride;
  const Dev& P = ctx->dev;
  const Fast& F = ctx->fast;
  cudaStream_t s = ctx->stream;
  const pbf_tuning& T = ctx->tune;
  const int g = blocks_for(n);
  // skippable launches: persistent grids
  const int gpc = std::min(grid_of(ctx, PBF_TUNE_DENSITY), ctx->pgrid_check);
  const int gpd = std::min(grid_of(ctx, PBF_TUNE_DELTA_P), ctx->pgrid_dp);
  const int bd = T.block[PBF_TUNE_DENSITY], bp = T.block[PBF_TUNE_DELTA_P];
  const float tol = ctx->params.residual_tol;
  const int iters = ctx->params.max_iterations > 0 ? ctx->params.max_iterations : 1;
  cudaMemsetAsync(ctx->state, 0, sizeof(pbf::SolveState), s);
  LearnIO io{nullptr, nullptr, nullptr, ctx->state, ctx->partials, 0, tol, 0};
  const pbf::MlpDev M = mlp_dev(ctx);
  {
    // the density family's shape (4 lanes x 128 threads when that family is staged)
    const int fl = T.staged[PBF_TUNE_DENSITY] ? 4 : T.lanes[PBF_TUNE_DENSITY];
    const int fb = T.staged[PBF_TUNE_DENSITY] ? kStageThreads : T.block[PBF_TUNE_DENSITY];
    with_lanes(fl, [&](auto gl) {
      Launch L(ctx, "warm_features");
      kl_features<decltype(gl)::value><<<blocks_for((size_t)n * fl, fb), fb, 0, s>>>(
          P, F, M, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->xl, ctx->velS, ctx->lamH, ctx->nudge, ctx->lamprevS,
          ctx->featb);
    });
  }
  {
    Launch L(ctx, "warm_mlp");
    kl_mlp_tc<true><<<mlp_tc_grid(ctx, n), pbf::tc::kThreads, 0, s>>>(M, n, ctx->featb, nullptr, ctx->xl, ctx->lamH,
                                                                 ctx->lamsumH, nullptr, ctx->err);
  }
  const TileIO tio = tile_io(ctx);
  if (T.staged[PBF_TUNE_DELTA_P]) {
    Launch L(ctx, "dp_update");
    ks_dp_update<SCORR, false, false><<<grid_of(ctx, PBF_TUNE_DELTA_P), kStageThreads, 0, s>>>(
        P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->pstS, ctx->posS, ctx->velS, ctx->state, nullptr, tio);
  } else {
    with_lanes(T.lanes[PBF_TUNE_DELTA_P], [&](auto gl) {
      Launch L(ctx, "dp_update");
      kf_dp_update<SCORR, false, false, decltype(gl)::value><<<grid_of(ctx, PBF_TUNE_DELTA_P), bp, 0, s>>>(
          P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->pstS, ctx->posS, ctx->velS, ctx->state, nullptr);
    });
  }
  if (!(tol > 0.0f)) {
    // A fixed count (residual_tol <= 0): max_iterations - 1 plain iterations
    // after the network's, no residual checks.  Each is the plain step's
    // density/lambda and delta-p pass; the latter adds its lambda to the
    // step's sum (the next step's feature).
    for (int r = 1; r < iters; ++r) {
      if (T.staged[PBF_TUNE_DENSITY]) {
        Launch L(ctx, "density_lambda");
        ks_density_lambda<kDlPlain><<<grid_of(ctx, PBF_TUNE_DENSITY), kStageThreads, 0, s>>>(
            P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->xl, ctx->velS, ctx->lamH, ctx->nudge, io, tio);
      } else {
        with_lanes(T.lanes[PBF_TUNE_DENSITY], [&](auto gl) {
          Launch L(ctx, "density_lambda");
          kf_density_lambda<kDlPlain, decltype(gl)::value><<<grid_of(ctx, PBF_TUNE_DENSITY), bd, 0, s>>>(
              P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->xl, ctx->velS, ctx->lamH, ctx->nudge, io);
        });
      }
      if (T.staged[PBF_TUNE_DELTA_P]) {
        Launch L(ctx, "dp_update");
        ks_dp_update<SCORR, false, false><<<grid_of(ctx, PBF_TUNE_DELTA_P), kStageThreads, 0, s>>>(
            P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->pstS, ctx->posS, ctx->velS, ctx->state, ctx->lamsumH,
            tio);
      } else {
        with_lanes(T.lanes[PBF_TUNE_DELTA_P], [&](auto gl) {
          Launch L(ctx, "dp_update");
          kf_dp_update<SCORR, false, false, decltype(gl)::value><<<grid_of(ctx, PBF_TUNE_DELTA_P), bp, 0, s>>>(
              P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->pstS, ctx->posS, ctx->velS, ctx->state, ctx->lamsumH);
        });
      }
    }
    Launch L(ctx, "update_velocities");
    k_update_v<<<g, kBlock, 0, s>>>(P, n, ctx->pstS, ctx->posS, ctx->velS);
    return;
  }
  // a residual check (final: the step's last, which only records) and a
  // plain position update, each skipping itself once the step is done.
  // Sampled checks (residual_sample > 1, direct density shapes): the check
  // estimates the residual from every S-th slot, and a plain density/lambda
  // pass, skipped once the step is done, precedes each position update.
  const int sample = ctx->params.residual_sample;
  const bool sampled = sample > 1 && !T.staged[PBF_TUNE_DENSITY];
  auto check = [&](cudaStream_t cs, const LearnIO& cio) {
    if (sampled) {
      with_lanes(T.lanes[PBF_TUNE_DENSITY], [&](auto gl) {
        constexpr int GL = decltype(gl)::value;
        Launch L(ctx, "residual_check");
        if (cio.loop.use)
          kl_residual_probe<GL, true><<<gpc, bd, 0, cs>>>(P, F, n, sample, st, ctx->nbr, ctx->cnt, ctx->pstS, cio);
        else
          kl_residual_probe<GL, false><<<gpc, bd, 0, cs>>>(P, F, n, sample, st, ctx->nbr, ctx->cnt, ctx->pstS, cio);
      });
      return;
    }
    if (T.staged[PBF_TUNE_DENSITY]) {
      Launch L(ctx, "residual_check");
      if (cio.loop.use)
        ks_density_lambda<kDlCheck, true><<<gpc, kStageThreads, 0, cs>>>(
            P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->xl, ctx->velS, ctx->lamH, ctx->nudge, cio, tio);
      else
        ks_density_lambda<kDlCheck, false><<<gpc, kStageThreads, 0, cs>>>(
            P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->xl, ctx->velS, ctx->lamH, ctx->nudge, cio, tio);
    } else {
      with_lanes(T.lanes[PBF_TUNE_DENSITY], [&](auto gl) {
        constexpr int GL = decltype(gl)::value;
        Launch L(ctx, "residual_check");
        if (cio.loop.use)
          kf_density_lambda<kDlCheck, GL, true><<<gpc, bd, 0, cs>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS,
                                                                    ctx->xl, ctx->velS, ctx->lamH, ctx->nudge, cio);
        else
          kf_density_lambda<kDlCheck, GL, false><<<gpc, bd, 0, cs>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS,
                                                                     ctx->xl, ctx->velS, ctx->lamH, ctx->nudge, cio);
      });
    }
  };
  auto update = [&](cudaStream_t cs) {
    if (sampled) {  // lambda of the iteration, skipped once the step is done
      with_lanes(T.lanes[PBF_TUNE_DENSITY], [&](auto gl) {
        Launch L(ctx, "density_lambda");
        kf_density_lambda<kDlPlain, decltype(gl)::value, false, true><<<gpc, bd, 0, cs>>>(
            P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->xl, ctx->velS, ctx->lamH, ctx->nudge, io);
      });
    }
    if (T.staged[PBF_TUNE_DELTA_P]) {
      Launch L(ctx, "dp_update");
      ks_dp_update<SCORR, false, true><<<gpd, kStageThreads, 0, cs>>>(
          P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->pstS, ctx->posS, ctx->velS, ctx->state, ctx->lamsumH, tio);
    } else {
      with_lanes(T.lanes[PBF_TUNE_DELTA_P], [&](auto gl) {
        Launch L(ctx, "dp_update");
        kf_dp_update<SCORR, false, true, decltype(gl)::value><<<gpd, bp, 0, cs>>>(
            P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->pstS, ctx->posS, ctx->velS, ctx->state, ctx->lamsumH);
      });
    }
  };
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cap);
  if (cap == cudaStreamCaptureStatusActive && iters > 1) {
    // Captured into the step's graph: the plain iterations become a WHILE
    // node whose body is (check, update) and whose condition the check sets
    // (SolveLoop), so a converged step launches nothing more; the final
    // check follows the node.  The node enters its loop on every graph launch
    // and only the body's check ends it, so a node whose body was not
    // captured whole must never run: any failure here marks the capture
    // failed, and pbf_step discards the graph instead of launching it.
    bool ok = false;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaGraphConditionalHandle h = 0;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (cudaStreamGetCaptureInfo(s, &cap, nullptr, &graph, &deps, &ndeps) == cudaSuccess &&
        cudaGraphConditionalHandleCreate(&h, graph, 1u, cudaGraphCondAssignDefault) == cudaSuccess &&
        (cp.conditional.handle = h, cudaGraphAddNode(&node, graph, deps, ndeps, &cp) == cudaSuccess)) {
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      if (cudaStreamBeginCaptureToGraph(ctx->side, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
          cudaSuccess) {
        LearnIO lio = io;
        lio.final_check = 0;
        lio.loop = pbf::SolveLoop{h, 1, iters};
        check(ctx->side, lio);
        update(ctx->side);
        const bool launched = cudaPeekAtLastError() == cudaSuccess;
        const bool ended = cudaStreamEndCapture(ctx->side, &body) == cudaSuccess;
        ok = launched && ended &&
             cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies) == cudaSuccess;
      }
    }
    if (!ok) ctx->capture_failed = true;
    LearnIO fio = io;
    fio.final_check = 1;
    check(s, fio);
  } else {
    for (int r = 1; r <= iters; ++r) {
      const bool final_check = r == iters;
      io.final_check = final_check ? 1 : 0;
      check(s, io);
      if (final_check) break;
      update(s);
    }
  }
  Launch L(ctx, "update_velocities");
  k_update_v<<<g, kBlock, 0, s>>>(P, n, ctx->pstS, ctx->posS, ctx->velS);
}

template <bool X, bool SCORR>
void launch_step_t(pbf_ctx* ctx) {
  const int n = (int)ctx->n;
  const size_t st = ctx->lstride;
  const Dev& P = ctx->dev;
  cudaStream_t s = ctx->stream;
  const int g = blocks_for(n);
  cudaMemsetAsync(ctx->cell_count, 0, sizeof(uint32_t) * ((size_t)ctx->nbins + 1), s);  // + the crowded flag
  {
    Launch L(ctx, "ext_predict_hash");
    k_ext_predict_hash<<<g, kBlock, 0, s>>>(P, n, ctx->posH, ctx->velH, ctx->pstH, ctx->origH, ctx->key,
                                            ctx->cell_count, ctx->key_ref, ctx->pairs, ctx->err);
  }
  launch_sort_to_pairs(ctx);
  {
    Launch L(ctx, "reorder");
    const bool keep = !X && (ctx->recording || ctx->params.solver == 1);
    k_reorder<false><<<g, kBlock, 0, s>>>(n, ctx->sorted, ctx->key, ctx->posH, ctx->pstH, ctx->velH, nullptr,
                                          keep ? ctx->lamsumH : nullptr, ctx->posS, ctx->pstS, ctx->velS, nullptr,
                                          keep ? ctx->lamprevS : nullptr, ctx->origS, ctx->keyH);
  }
  if (!X && !SCORR && persist_on(ctx)) {
    launch_persistent(ctx);
    return;
  }
  launch_fill(ctx, ctx->pstS);
  const int K = ctx->params.solve_steps;
  const Fast& F = ctx->fast;
  const pbf_tuning& T = ctx->tune;
  if (!X && ctx->params.solver == 1) {
    launch_learned_solve<SCORR>(ctx);
  } else {
  LearnIO io{ctx->feats, ctx->lamsumH, ctx->lamprevS, ctx->state, nullptr, 0, 0.0f, 0};
  for (int it = 0; it < K; ++it) {
    io.first = it == 0;
    if (X) cudaMemsetAsync(ctx->nudge, 0, sizeof(uint32_t), s);
    {
      Launch L(ctx, "density_lambda");
      if (X)
        k_density_lambda<X><<<g, kBlock, 0, s>>>(P, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->xl, ctx->velS,
                                                 ctx->lamH, ctx->nudge);
      else if (T.staged[PBF_TUNE_DENSITY]) {
        const int gd = grid_of(ctx, PBF_TUNE_DENSITY);
        if (ctx->recording)
          ks_density_lambda<kDlRecord><<<gd, kStageThreads, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS,
                                                                    ctx->xl, ctx->velS, ctx->lamH, ctx->nudge, io,
                                                                    tile_io(ctx));
        else
          ks_density_lambda<kDlPlain><<<gd, kStageThreads, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS,
                                                                   ctx->xl, ctx->velS, ctx->lamH, ctx->nudge, io,
                                                                   tile_io(ctx));
      } else
        with_lanes(T.lanes[PBF_TUNE_DENSITY], [&](auto gl) {
          constexpr int GL = decltype(gl)::value;
          const int gd = grid_of(ctx, PBF_TUNE_DENSITY), bd = T.block[PBF_TUNE_DENSITY];
          if (ctx->recording)
            kf_density_lambda<kDlRecord, GL><<<gd, bd, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->xl,
                                                               ctx->velS, ctx->lamH, ctx->nudge, io);
          else
            kf_density_lambda<kDlPlain, GL><<<gd, bd, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->xl,
                                                              ctx->velS, ctx->lamH, ctx->nudge, io);
        });
    }
    if (X) {
      Launch L(ctx, "lambda_fixup");
      k_lambda_fixup<X><<<g, kBlock, 0, s>>>(P, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->velS, ctx->lamH,
                                             ctx->nudge);
    }
    Launch L(ctx, "dp_update");
    const bool last = it == K - 1;
    if (X) {
      if (last)
        k_dp_update<X, SCORR, true><<<g, kBlock, 0, s>>>(P, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->pstS,
                                                         ctx->posS, ctx->velS, ctx->lamH, ctx->nudge);
      else
        k_dp_update<X, SCORR, false><<<g, kBlock, 0, s>>>(P, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->pstS,
                                                          ctx->posS, ctx->velS, ctx->lamH, ctx->nudge);
    } else if (T.staged[PBF_TUNE_DELTA_P]) {
      const int gd = grid_of(ctx, PBF_TUNE_DELTA_P);
      if (last)
        ks_dp_update<SCORR, true, false><<<gd, kStageThreads, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl,
                                                                      ctx->pstS, ctx->posS, ctx->velS, ctx->state,
                                                                      nullptr, tile_io(ctx));
      else
        ks_dp_update<SCORR, false, false><<<gd, kStageThreads, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl,
                                                                       ctx->pstS, ctx->posS, ctx->velS, ctx->state,
                                                                       nullptr, tile_io(ctx));
    } else {
      with_lanes(T.lanes[PBF_TUNE_DELTA_P], [&](auto gl) {
        constexpr int GL = decltype(gl)::value;
        const int gd = grid_of(ctx, PBF_TUNE_DELTA_P), bd = T.block[PBF_TUNE_DELTA_P];
        if (last)
          kf_dp_update<SCORR, true, false, GL><<<gd, bd, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->pstS,
                                                                 ctx->posS, ctx->velS, ctx->state, nullptr);
        else
          kf_dp_update<SCORR, false, false, GL><<<gd, bd, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl,
                                                                  ctx->pstS, ctx->posS, ctx->velS, ctx->state, nullptr);
      });
    }
  }
  }
  if (K == 0 && !(!X && ctx->params.solver == 1)) {
    Launch L(ctx, "update_velocities");
    k_update_v<<<g, kBlock, 0, s>>>(P, n, ctx->pstS, ctx->posS, ctx->velS);
  }
  if (ctx->params.gamma != 0.0f) {
    {
      Launch L(ctx, "color_field");
      k_color<X><<<g, kBlock, 0, s>>>(P, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->velS, ctx->scrH);
    }
    Launch L(ctx, "surface_tension");
    k_surface<<<g, kBlock, 0, s>>>(P, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->scrH, ctx->velS);
  }
  if (X) {
    {
      Launch L(ctx, "viscosity");
      k_viscosity<X, false><<<g, kBlock, 0, s>>>(P, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->velS, ctx->velT,
                                                 nullptr, nullptr, nullptr, nullptr);
    }
    {
      Launch L(ctx, "vorticity");
      k_vorticity<X><<<g, kBlock, 0, s>>>(P, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->velT, ctx->scrH, ctx->xl);
    }
    {
      Launch L(ctx, "apply_vorticity");
      k_apply_vorticity<X, true><<<g, kBlock, 0, s>>>(P, n, st, ctx->nbr, ctx->cnt, ctx->xl, nullptr, ctx->scrH,
                                                      ctx->velT);
    }
    Launch L(ctx, "viscosity_final");
    k_viscosity<X, true><<<g, kBlock, 0, s>>>(P, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->velT, ctx->velH,
                                              ctx->posH, ctx->pstH, ctx->origS, ctx->origH);
  } else {
    const TileIO tio = tile_io(ctx);
    const int gv = grid_of(ctx, PBF_TUNE_VISCOSITY), bv = T.block[PBF_TUNE_VISCOSITY];
    if (T.staged[PBF_TUNE_VISCOSITY]) {
      Launch L(ctx, "viscosity");
      ks_viscosity<false><<<gv, kStageThreads, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->velS,
                                                       ctx->velT, nullptr, nullptr, nullptr, nullptr, tio);
    } else {
      with_lanes(T.lanes[PBF_TUNE_VISCOSITY], [&](auto gl) {
        Launch L(ctx, "viscosity");
        kf_viscosity<false, decltype(gl)::value><<<gv, bv, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS,
                                                                   ctx->velS, ctx->velT, nullptr, nullptr, nullptr,
                                                                   nullptr, ctx->wvis);
      });
    }
    if (T.staged[PBF_TUNE_VORTICITY]) {
      Launch L(ctx, "vorticity");
      ks_vorticity<<<grid_of(ctx, PBF_TUNE_VORTICITY), kStageThreads, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt,
                                                                               ctx->pstS, ctx->velT, ctx->scrH,
                                                                               ctx->xl, tio);
    } else {
      with_lanes(T.lanes[PBF_TUNE_VORTICITY], [&](auto gl) {
        Launch L(ctx, "vorticity");
        kf_vorticity<decltype(gl)::value><<<grid_of(ctx, PBF_TUNE_VORTICITY), T.block[PBF_TUNE_VORTICITY], 0, s>>>(
            P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->velT, ctx->scrH, ctx->xl);
      });
    }
    if (T.staged[PBF_TUNE_APPLY_VORTICITY]) {
      Launch L(ctx, "apply_vorticity");
      ks_apply_vorticity<<<grid_of(ctx, PBF_TUNE_APPLY_VORTICITY), kStageThreads, 0, s>>>(
          P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->scrH, ctx->velT, tio);
    } else {
      with_lanes(T.lanes[PBF_TUNE_APPLY_VORTICITY], [&](auto gl) {
        Launch L(ctx, "apply_vorticity");
        kf_apply_vorticity<decltype(gl)::value>
            <<<grid_of(ctx, PBF_TUNE_APPLY_VORTICITY), T.block[PBF_TUNE_APPLY_VORTICITY], 0, s>>>(
                P, F, n, st, ctx->nbr, ctx->cnt, ctx->xl, ctx->scrH, ctx->velT);
      });
    }
    if (T.staged[PBF_TUNE_VISCOSITY]) {
      Launch L(ctx, "viscosity_final");
      ks_viscosity<true><<<gv, kStageThreads, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS, ctx->velT,
                                                      ctx->velH, ctx->posH, ctx->pstH, ctx->origS, ctx->origH, tio);
    } else {
      with_lanes(T.lanes[PBF_TUNE_VISCOSITY], [&](auto gl) {
        Launch L(ctx, "viscosity_final");
        kf_viscosity<true, decltype(gl)::value><<<gv, bv, 0, s>>>(P, F, n, st, ctx->nbr, ctx->cnt, ctx->pstS,
                                                                  ctx->velT, ctx->velH, ctx->posH, ctx->pstH,
                                                                  ctx->origS, ctx->origH, ctx->wvis);
      });
    }
  }
}

void launch_step(pbf_ctx* ctx) {
  const bool X = ctx->params.exact_math != 0, SC = ctx->params.scorr_k > 0.0f;
  if (X) {
    if (SC) launch_step_t<true, true>(ctx); else launch_step_t<true, false>(ctx);
  } else {
    if (SC) launch_step_t<false, true>(ctx); else launch_step_t<false, false>(ctx);
  }
}

int launches_per_step(const pbf_ctx* ctx) {
  // kernels only (the memsets are not), as launched eagerly (a captured
  // learned step runs its plain iterations in a conditional graph node and
  // launches fewer once converged): ext/predict/hash + 3 scan + radix
  // passes x (histogram, 3 scan, scatter) + reorder + runs + fill + [fast
  // math: fill redo] + K x (density/lambda, [exact: lambda fix-up], delta-p)
  // + (K==0: velocity) + 2 if gamma + 4 (visc, vort, apply, visc)
  const int sort = 5 * ctx->radix_passes;
  const int fill = ctx->params.exact_math ? 2 : 3;  // runs, fill, [redo]
  if (persist_on(ctx)) return 1 + 3 + sort + 1 + fill + 1;  // ... reorder, runs, fill, redo, the persistent step
  const int K = ctx->params.solve_steps;
  const int tail = (ctx->params.gamma != 0.0f ? 2 : 0) + 4;
  if (ctx->params.solver == 1 && !ctx->params.exact_math && !(ctx->params.residual_tol > 0.0f)) {
    // learned, a fixed count: warm iteration (features, network, delta-p) + (iters-1) x (density, delta-p)
    // + velocity
    const int it = ctx->params.max_iterations > 0 ? ctx->params.max_iterations : 1;
    return 1 + 3 + sort + 1 + fill + 3 + 2 * (it - 1) + 1 + tail;
  }
  if (ctx->params.solver == 1 && !ctx->params.exact_math) {
    // learned: warm iteration (features, network, delta-p) + (iters-1) x (check, [sampled checks:
    // density/lambda,] delta-p) + final check + velocity
    const int it = ctx->params.max_iterations > 0 ? ctx->params.max_iterations : 1;
    const bool sampled = ctx->params.residual_sample > 1 && !ctx->tune.staged[PBF_TUNE_DENSITY];
    return 1 + 3 + sort + 1 + fill + 3 + (sampled ? 3 : 2) * (it - 1) + 1 + 1 + tail;
  }
  const int per_iter = ctx->params.exact_math ? 3 : 2;
  return 1 + 3 + sort + 1 + fill + per_iter * K + (K == 0 ? 1 : 0) + tail;
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

const char* pbf_create_error(void) { return g_create_error.c_str(); }
const char* pbf_last_error(const pbf_ctx* ctx) { return ctx ? ctx->error.c_str() : g_create_error.c_str(); }

static int create_ctx(const pbf_params* p, size_t capacity, const pbf_scene* scenes, int nscenes, pbf_ctx** out) {
  pbf_ctx* ctx = nullptr;
  if (!p || !out) return fail(nullptr, PBF_ERR_ARG, "null argument");
  *out = nullptr;
  if (capacity == 0 || capacity >= (size_t)1 << 31)
    return fail(nullptr, PBF_ERR_ARG, "capacity must be in [1, 2^31)");
  ctx = new pbf_ctx();
  ctx->params = *p;
  if (scenes) ctx->scenes.assign(scenes, scenes + nscenes);
  int rc = scenes ? make_dev_batch(ctx, *p, ctx->scenes, ctx->dev, ctx->regions, ctx->scene_first)
                  : make_dev(ctx, *p, ctx->dev, ctx->dims);
  if (rc) {
    g_create_error = ctx->error;
    delete ctx;
    return rc;
  }
  ctx->fast = pbf::make_fast(ctx->dev);
  ctx->capacity = capacity;
  ctx->nbins = ctx->dev.nbins;
  ctx->nbins_cap = ctx->nbins;
  ctx->radix_passes = radix_passes_for(ctx->nbins);
  ctx->nscan_parts = (int)(((size_t)ctx->nbins + 1 + kScanTile - 1) / kScanTile);
  auto bail = [&](int code) {
    g_create_error = ctx->error;
    pbf_destroy(ctx);
    return code;
  };
  if (cudaGetDevice(&ctx->device) != cudaSuccess) {
    fail(ctx, PBF_ERR_CUDA, "no CUDA device");
    return bail(PBF_ERR_CUDA);
  }
  {
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device) == cudaSuccess && sms > 0)
      ctx->sms = sms;
    if (cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxBlocksPerMultiprocessor, ctx->device) != cudaSuccess ||
        per_sm <= 0)
      per_sm = 32;
    ctx->partials_cap = ctx->sms * per_sm;
    if ((rc = update_shapes(ctx))) return bail(rc);
  }
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking) != cudaSuccess) {
    fail(ctx, PBF_ERR_CUDA, "cudaStreamCreate failed");
    return bail(PBF_ERR_CUDA);
  }
  const size_t C = capacity;
  ctx->lstride = list_stride(p->neighbor_cap);
  ctx->lstride_cap = ctx->lstride;
  const size_t cap = ctx->lstride;
  if ((rc = dalloc(ctx, &ctx->posH, C)) || (rc = dalloc(ctx, &ctx->pstH, C)) || (rc = dalloc(ctx, &ctx->velH, C)) ||
      (rc = dalloc(ctx, &ctx->scrH, C)) || (rc = dalloc(ctx, &ctx->posS, C)) || (rc = dalloc(ctx, &ctx->pstS, C + 1)) ||
      (rc = dalloc(ctx, &ctx->velS, C + 1)) || (rc = dalloc(ctx, &ctx->scrS, C)) || (rc = dalloc(ctx, &ctx->xl, C + 1)) ||
      (rc = dalloc(ctx, &ctx->velT, C + 1)) || (rc = dalloc(ctx, &ctx->lamH, C)) || (rc = dalloc(ctx, &ctx->lamS, C)) ||
      (rc = dalloc(ctx, &ctx->origH, C)) || (rc = dalloc(ctx, &ctx->origS, C)) || (rc = dalloc(ctx, &ctx->key, C)) ||
      (rc = dalloc(ctx, &ctx->key_ref, C)) || (rc = dalloc(ctx, &ctx->key_alt, C)) ||
      (rc = dalloc(ctx, &ctx->keyH, C)) || (rc = dalloc(ctx, &ctx->run_end, C)) ||
      (rc = dalloc(ctx, &ctx->radix_hist, radix_entries(C))) ||
      (rc = dalloc(ctx, &ctx->radix_off, radix_entries(C) + 1)) ||
      (rc = dalloc(ctx, &ctx->radix_parts, (radix_entries(C) + 1 + kScanTile - 1) / kScanTile)) ||
      (rc = dalloc(ctx, &ctx->cell_count, (size_t)ctx->nbins + 1)) ||
      (rc = dalloc(ctx, &ctx->cell_start, (size_t)ctx->nbins + 1)) ||
      (rc = dalloc(ctx, &ctx->scan_part, (size_t)ctx->nscan_parts)) || (rc = dalloc(ctx, &ctx->err, 1)) ||
      (rc = dalloc(ctx, &ctx->nudge, 1)) ||
      (rc = dalloc(ctx, &ctx->pairs, C)) || (rc = dalloc(ctx, &ctx->pairs_sorted, C)) || (rc = dalloc(ctx, &ctx->nbr, pbf::list_entries(C, cap))) ||
      (rc = dalloc(ctx, &ctx->seg, C * kSegWords)) || (rc = dalloc(ctx, &ctx->fill_words, kFillWords)) ||
      (rc = dalloc(ctx, &ctx->redo_queue, C)) ||
            (rc = dalloc(ctx, &ctx->cnt, C)) || (rc = dalloc(ctx, &ctx->stage, 6 * C)) ||
      (rc = dalloc(ctx, &ctx->stage_i, std::max(C * cap + C, pbf::list_entries(C, cap)))) ||
      (rc = dalloc(ctx, &ctx->acc, 8)) ||
      (rc = dalloc(ctx, &ctx->maxerr, 1)) || (rc = dalloc(ctx, &ctx->hits, 1)) ||
      (rc = dalloc(ctx, &ctx->lamsumH, C)) || (rc = dalloc(ctx, &ctx->lamprevS, C)) ||
      (rc = dalloc(ctx, &ctx->featb, C * pbf::kMlpInPad)) ||
      (rc = dalloc(ctx, &ctx->tile_nruns, (C + kTile - 1) / kTile)) ||
      (rc = dalloc(ctx, &ctx->tile_total, (C + kTile - 1) / kTile)) ||
      (rc = dalloc(ctx, &ctx->tile_runs, (C + kTile - 1) / kTile * kTileRuns)) ||
      (rc = dalloc(ctx, &ctx->nbr16, C * cap)) ||
      (rc = dalloc(ctx, &ctx->state, 1)) || (rc = dalloc(ctx, &ctx->partials, (size_t)ctx->partials_cap)) ||
      (rc = dalloc(ctx, &ctx->mlp_params, pbf::kMlpParams)) ||
      (rc = dalloc(ctx, &ctx->mlp_grad, pbf::kMlpParams)) || (rc = dalloc(ctx, &ctx->mlp_m, pbf::kMlpParams)) ||
      (rc = dalloc(ctx, &ctx->mlp_v, pbf::kMlpParams)) || (rc = dalloc(ctx, &ctx->mlp_norm, 32)) ||
      (rc = dalloc(ctx, &ctx->mlp_loss, 1)) || (rc = dalloc(ctx, &ctx->w1b, pbf::kMlpH * pbf::kMlpInPad)) ||
      (rc = dalloc(ctx, &ctx->w2b, pbf::kMlpH * pbf::kMlpH)) || (rc = dalloc(ctx, &ctx->w2tb, pbf::kMlpH * pbf::kMlpH)))
    return bail(rc);
  ctx->wvis = reinterpret_cast<__half*>(ctx->stage_i);
  if (!ctx->scenes.empty() &&
      ((rc = dalloc(ctx, &ctx->d_regions, ctx->regions.size())) ||
       (rc = dalloc(ctx, &ctx->d_scene_first, ctx->scene_first.size())) || (rc = upload_scenes(ctx))))
    return bail(rc);
  if (cudaMemsetAsync(ctx->lamsumH, 0, C * sizeof(float), ctx->stream) != cudaSuccess ||
      cudaMemsetAsync(ctx->state, 0, sizeof(pbf::SolveState), ctx->stream) != cudaSuccess) {
    fail(ctx, PBF_ERR_CUDA, "initialisation failed");
    return bail(PBF_ERR_CUDA);
  }
  // the first fill walks in slot order (the byte sets word kFillSlotOrder to 1)
  if (cudaMemsetAsync(ctx->err, 0, sizeof(uint32_t), ctx->stream) != cudaSuccess ||
      cudaMemsetAsync(ctx->fill_words, 0, kFillWords * sizeof(uint32_t), ctx->stream) != cudaSuccess ||
      cudaMemsetAsync(ctx->fill_words + kFillSlotOrder, 1, 1, ctx->stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    fail(ctx, PBF_ERR_CUDA, "initialisation failed");
    return bail(PBF_ERR_CUDA);
  }
  *out = ctx;
  return PBF_OK;
}

int pbf_create(const pbf_params* p, size_t capacity, pbf_ctx** out) {
  return create_ctx(p, capacity, nullptr, 0, out);
}

int pbf_create_batch(const pbf_params* p, const pbf_scene* scenes, int nscenes, pbf_ctx** out) {
  if (!scenes || nscenes < 1) return fail(nullptr, PBF_ERR_ARG, "a batch needs at least one scene");
  size_t total = 0;
  for (int i = 0; i < nscenes; ++i) total += scenes[i].count;
  if (total == 0) return fail(nullptr, PBF_ERR_ARG, "a batch needs at least one particle");
  return create_ctx(p, total, scenes, nscenes, out);
}

void pbf_destroy(pbf_ctx* ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  drop_graphs(ctx);
  for (auto& m : ctx->marks) {
    cudaEventDestroy(m.start);
    cudaEventDestroy(m.stop);
  }
  for (void* p : ctx->allocations) cudaFree(p);
  if (ctx->side) cudaStreamDestroy(ctx->side);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int pbf_set_params(pbf_ctx* ctx, const pbf_params* p) {
  if (!ctx || !p) return PBF_ERR_ARG;
  Dev d;
  int64_t dims[3] = {0, 0, 0};
  std::vector<pbf::Region> regions;
  std::vector<uint32_t> first;
  const bool batch = !ctx->scenes.empty();
  int rc = batch ? make_dev_batch(ctx, *p, ctx->scenes, d, regions, first) : make_dev(ctx, *p, d, dims);
  if (rc) return rc;
  const size_t lstride = list_stride(p->neighbor_cap);
  if (d.nbins > ctx->nbins_cap || lstride > ctx->lstride_cap)
    return fail(ctx, PBF_ERR_PARAMS, "new parameters need a larger grid or neighbor cap than allocated");
  if (d.nbins != ctx->nbins || p->neighbor_cap != ctx->params.neighbor_cap || d.s != ctx->dev.s)
    ctx->lists_valid = false;
  ctx->params = *p;
  ctx->dev = d;
  ctx->fast = pbf::make_fast(d);
  ctx->lstride = lstride;
  std::memcpy(ctx->dims, dims, sizeof(dims));
  ctx->nbins = d.nbins;
  ctx->radix_passes = radix_passes_for(ctx->nbins);
  ctx->nscan_parts = (int)(((size_t)ctx->nbins + 1 + kScanTile - 1) / kScanTile);
  if (batch) {
    ctx->regions = regions;
    ctx->scene_first = first;
    if ((rc = upload_scenes(ctx))) return rc;
  }
  drop_graphs(ctx);
  return PBF_OK;
}

int pbf_get_params(const pbf_ctx* ctx, pbf_params* p) {
  if (!ctx || !p) return PBF_ERR_ARG;
  *p = ctx->params;
  return PBF_OK;
}

size_t pbf_count(const pbf_ctx* ctx) { return ctx ? ctx->n : 0; }
int64_t pbf_num_bins(const pbf_ctx* ctx) { return ctx ? ctx->nbins : 0; }

int pbf_upload(pbf_ctx* ctx, const float* x, const float* v, size_t n) {
  if (!ctx || (!x && n)) return ctx ? fail(ctx, PBF_ERR_ARG, "null positions") : PBF_ERR_ARG;
  if (n > ctx->capacity)
    return fail(ctx, PBF_ERR_CAPACITY, "Not enough capacity: %zu particles > capacity %zu", n, ctx->capacity);
  if (!ctx->scenes.empty() && n != ctx->scene_first.back())
    return fail(ctx, PBF_ERR_ARG, "a batch of %zu scenes takes exactly %u particles (its scenes' counts), got %zu",
                ctx->scenes.size(), ctx->scene_first.back(), n);
  if (n != ctx->n) drop_graphs(ctx);
  ctx->n = n;
  ctx->lists_valid = false;
  if (int rc = reset_fill_order(ctx)) return rc;
  if (n == 0) return PBF_OK;
  float* dx = ctx->stage;
  float* dv = ctx->stage + 3 * ctx->capacity;
  CK(cudaMemcpyAsync(dx, x, n * 3 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  if (v) CK(cudaMemcpyAsync(dv, v, n * 3 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ctx->lamsumH, 0, n * sizeof(float), ctx->stream));  // no lambda history yet
  k_upload<<<blocks_for(n), kBlock, 0, ctx->stream>>>((int)n, dx, v ? dv : nullptr, ctx->posH, ctx->pstH,
                                                      ctx->velH, ctx->scrH, ctx->lamH, ctx->origH, ctx->pstS,
                                                      ctx->xl, ctx->velS, ctx->velT);
  return check_launch(ctx, "upload");
}

static int get_array_dev(pbf_ctx* ctx, int which, float* dst) {
  const int n = (int)ctx->n, g = blocks_for(n);
  switch (which) {
    case PBF_ARRAY_POSITIONS: k_unpermute_vec<<<g, kBlock, 0, ctx->stream>>>(n, ctx->posH, ctx->origH, dst); break;
    case PBF_ARRAY_POSITION_STARS: k_unpermute_vec<<<g, kBlock, 0, ctx->stream>>>(n, ctx->pstH, ctx->origH, dst); break;
    case PBF_ARRAY_VELOCITIES: k_unpermute_vec<<<g, kBlock, 0, ctx->stream>>>(n, ctx->velH, ctx->origH, dst); break;
    case PBF_ARRAY_SCRATCH: k_unpermute_vec<<<g, kBlock, 0, ctx->stream>>>(n, ctx->scrH, ctx->origH, dst); break;
    case PBF_ARRAY_DENSITIES: k_unpermute_w<<<g, kBlock, 0, ctx->stream>>>(n, ctx->velH, nullptr, ctx->origH, dst); break;
    case PBF_ARRAY_LAMBDAS: k_unpermute_w<<<g, kBlock, 0, ctx->stream>>>(n, nullptr, ctx->lamH, ctx->origH, dst); break;
    default: return fail(ctx, PBF_ERR_ARG, "unknown array %d", which);
  }
  return check_launch(ctx, "unpermute");
}

int pbf_get_array(pbf_ctx* ctx, int which, float* host_out) {
  if (!ctx || !host_out) return PBF_ERR_ARG;
  if (ctx->n == 0) return PBF_OK;
  const bool vec = which <= PBF_ARRAY_SCRATCH;
  int rc = get_array_dev(ctx, which, ctx->stage);
  if (rc) return rc;
  CK(cudaMemcpyAsync(host_out, ctx->stage, ctx->n * (vec ? 3 : 1) * sizeof(float), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

int pbf_set_array(pbf_ctx* ctx, int which, const float* host_in) {
  if (!ctx || !host_in) return PBF_ERR_ARG;
  if (ctx->n == 0) return PBF_OK;
  const int n = (int)ctx->n, g = blocks_for(n);
  const bool vec = which <= PBF_ARRAY_SCRATCH;
  CK(cudaMemcpyAsync(ctx->stage, host_in, ctx->n * (vec ? 3 : 1) * sizeof(float), cudaMemcpyHostToDevice,
                     ctx->stream));
  switch (which) {
    case PBF_ARRAY_POSITIONS: k_permute_vec_in<<<g, kBlock, 0, ctx->stream>>>(n, ctx->stage, ctx->origH, ctx->posH); break;
    case PBF_ARRAY_POSITION_STARS: k_permute_vec_in<<<g, kBlock, 0, ctx->stream>>>(n, ctx->stage, ctx->origH, ctx->pstH); break;
    case PBF_ARRAY_VELOCITIES: k_permute_vec_in<<<g, kBlock, 0, ctx->stream>>>(n, ctx->stage, ctx->origH, ctx->velH); break;
    case PBF_ARRAY_SCRATCH: k_permute_vec_in<<<g, kBlock, 0, ctx->stream>>>(n, ctx->stage, ctx->origH, ctx->scrH); break;
    case PBF_ARRAY_DENSITIES: k_permute_w_in<<<g, kBlock, 0, ctx->stream>>>(n, ctx->stage, ctx->origH, ctx->velH, nullptr); break;
    case PBF_ARRAY_LAMBDAS: k_permute_w_in<<<g, kBlock, 0, ctx->stream>>>(n, ctx->stage, ctx->origH, nullptr, ctx->lamH); break;
    default: return fail(ctx, PBF_ERR_ARG, "unknown array %d", which);
  }
  int rc = check_launch(ctx, "set_array");
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

// ---- growing the particle set ----
int pbf_add_particles(pbf_ctx* ctx, const float* x, const float* v, size_t k) {
  if (!ctx || (!x && k)) return ctx ? fail(ctx, PBF_ERR_ARG, "null positions") : PBF_ERR_ARG;
  if (!ctx->scenes.empty()) return fail(ctx, PBF_ERR_STATE, "the scenes of a batch have fixed particle counts");
  if (k == 0) return PBF_OK;
  if (ctx->n + k > ctx->capacity)
    return fail(ctx, PBF_ERR_CAPACITY, "Not enough capacity: %zu particles > capacity %zu", ctx->n + k,
                ctx->capacity);
  float* dx = ctx->stage;
  float* dv = ctx->stage + 3 * ctx->capacity;
  CK(cudaMemcpyAsync(dx, x, k * 3 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  if (v) CK(cudaMemcpyAsync(dv, v, k * 3 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  k_append<<<blocks_for(k), kBlock, 0, ctx->stream>>>((int)ctx->n, (int)k, dx, v ? dv : nullptr, ctx->posH,
                                                      ctx->pstH, ctx->velH, ctx->scrH, ctx->lamH, ctx->lamsumH,
                                                      ctx->origH, ctx->pstS, ctx->xl, ctx->velS, ctx->velT);
  if (int rc = check_launch(ctx, "add_particles")) return rc;
  CK(cudaStreamSynchronize(ctx->stream));  // the host buffers may go once this returns
  ctx->n += k;
  ctx->lists_valid = false;
  drop_graphs(ctx);
  return PBF_OK;
}

int pbf_construct_fluid(pbf_ctx* ctx, const float fluid_min[3], const float fluid_max[3], const float velocity[3],
                        size_t* added) {
  if (added) *added = 0;
  if (!ctx || !fluid_min || !fluid_max) return PBF_ERR_ARG;
  int64_t d[3];
  if (int rc = pbf_lattice_dims(fluid_min, fluid_max, ctx->params.particle_rest_spacing, d))
    return fail(ctx, rc, "particle_rest_spacing must be > 0");
  const size_t k = (size_t)(d[0] * d[1] * d[2]);
  if (k == 0) return PBF_OK;
  if (ctx->n + k > ctx->capacity)
    return fail(ctx, PBF_ERR_CAPACITY, "Not enough capacity: %zu particles > capacity %zu", ctx->n + k,
                ctx->capacity);
  std::vector<float> x(3 * k), v(3 * k, 0.0f);
  if (int rc = pbf_build_lattice(fluid_min, d, ctx->params.particle_rest_spacing, 0.0f, 0, x.data()))
    return fail(ctx, rc, "lattice construction failed");
  if (velocity)
    for (size_t i = 0; i < k; ++i)
      for (int a = 0; a < 3; ++a) v[3 * i + a] = velocity[a];
  if (int rc = pbf_add_particles(ctx, x.data(), v.data(), k)) return rc;
  if (added) *added = k;
  return PBF_OK;
}

uint64_t pbf_step_count(const pbf_ctx* ctx) { return ctx ? ctx->steps_done : 0; }

// ---- the state file (output frames, checkpoints) ----
namespace {
constexpr char kStateMagic[8] = {'P', 'B', 'F', 'S', 'T', 'A', 'T', 'E'};
constexpr uint32_t kStateVersion = 1;
struct StateHeader {
  char magic[8];
  uint32_t version;
  uint32_t params_bytes;
  uint64_t n;
  uint64_t steps;
  uint32_t flags;  // bit 0: the learned warm start's network follows the arrays
  uint32_t reserved;
  pbf_tuning tuning;
  uint32_t reserved2;  // the header is 104 bytes, a multiple of 8
};
static_assert(sizeof(StateHeader) == 104, "state file header layout");
struct FileCloser {
  FILE* f;
  ~FileCloser() {
    if (f) std::fclose(f);
  }
};
}  // namespace

int pbf_save_state(pbf_ctx* ctx, const char* path) {
  if (!ctx || !path) return PBF_ERR_ARG;
  const size_t n = ctx->n;
  std::vector<float> x(3 * n), v(3 * n), rho(n), lam(n), hist(n);
  if (n) {
    if (int rc = pbf_download(ctx, x.data(), v.data(), rho.data(), lam.data())) return rc;
    k_unpermute_w<<<blocks_for(n), kBlock, 0, ctx->stream>>>((int)n, nullptr, ctx->lamsumH, ctx->origH, ctx->stage);
    if (int rc = check_launch(ctx, "save_state")) return rc;
    CK(cudaMemcpyAsync(hist.data(), ctx->stage, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  std::vector<float> net, norm;
  if (ctx->mlp_ready) {
    net.resize(pbf::kMlpParams);
    norm.resize(PBF_MLP_NORM);
    if (int rc = pbf_mlp_get(ctx, net.data(), norm.data())) return rc;
  }
  StateHeader h{};
  std::memcpy(h.magic, kStateMagic, 8);
  h.version = kStateVersion;
  h.params_bytes = (uint32_t)sizeof(pbf_params);
  h.n = n;
  h.steps = ctx->steps_done;
  h.flags = ctx->mlp_ready ? 1u : 0u;
  h.tuning = ctx->tune;
  FileCloser fc{std::fopen(path, "wb")};
  if (!fc.f) return fail(ctx, PBF_ERR_IO, "cannot open %s for writing", path);
  bool ok = std::fwrite(&h, sizeof(h), 1, fc.f) == 1 && std::fwrite(&ctx->params, sizeof(pbf_params), 1, fc.f) == 1;
  auto put = [&](const std::vector<float>& a) {
    if (ok && !a.empty()) ok = std::fwrite(a.data(), sizeof(float), a.size(), fc.f) == a.size();
  };
  put(x);
  put(v);
  put(rho);
  put(lam);
  put(hist);
  put(net);
  put(norm);
  if (!ok || std::fflush(fc.f) != 0) return fail(ctx, PBF_ERR_IO, "short write to %s", path);
  return PBF_OK;
}

int pbf_load_state(pbf_ctx* ctx, const char* path) {
  if (!ctx || !path) return PBF_ERR_ARG;
  FileCloser fc{std::fopen(path, "rb")};
  if (!fc.f) return fail(ctx, PBF_ERR_IO, "cannot open %s", path);
  StateHeader h{};
  pbf_params p{};
  if (std::fread(&h, sizeof(h), 1, fc.f) != 1 || std::memcmp(h.magic, kStateMagic, 8) != 0)
    return fail(ctx, PBF_ERR_IO, "%s is not a PBF state file", path);
  if (h.version != kStateVersion || h.params_bytes != sizeof(pbf_params))
    return fail(ctx, PBF_ERR_IO, "%s: state version %u / parameter block %u bytes, this library reads %u / %zu", path,
                h.version, h.params_bytes, kStateVersion, sizeof(pbf_params));
  if (std::fread(&p, sizeof(p), 1, fc.f) != 1) return fail(ctx, PBF_ERR_IO, "%s: truncated", path);
  if (h.n > ctx->capacity)
    return fail(ctx, PBF_ERR_CAPACITY, "Not enough capacity: %llu particles > capacity %zu",
                (unsigned long long)h.n, ctx->capacity);
  const size_t n = (size_t)h.n;
  std::vector<float> x(3 * n), v(3 * n), rho(n), lam(n), hist(n);
  bool ok = true;
  auto get = [&](std::vector<float>& a) {
    if (ok && !a.empty()) ok = std::fread(a.data(), sizeof(float), a.size(), fc.f) == a.size();
  };
  get(x);
  get(v);
  get(rho);
  get(lam);
  get(hist);
  std::vector<float> net, norm;
  if (h.flags & 1u) {
    net.resize(pbf::kMlpParams);
    norm.resize(PBF_MLP_NORM);
    get(net);
    get(norm);
  }
  if (!ok) return fail(ctx, PBF_ERR_IO, "%s: truncated", path);
  int rc;
  if ((rc = pbf_set_params(ctx, &p)) || (rc = pbf_set_tuning(ctx, &h.tuning)) ||
      (rc = pbf_upload(ctx, x.data(), v.data(), n)))
    return rc;
  if (n) {
    if ((rc = pbf_set_array(ctx, PBF_ARRAY_DENSITIES, rho.data())) ||
        (rc = pbf_set_array(ctx, PBF_ARRAY_LAMBDAS, lam.data())))
      return rc;
    // after an upload the slots are in reference order
    CK(cudaMemcpyAsync(ctx->lamsumH, hist.data(), n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  if ((h.flags & 1u) && (rc = pbf_mlp_set(ctx, net.data(), norm.data()))) return rc;
  ctx->steps_done = h.steps;
  return PBF_OK;
}

int pbf_download(pbf_ctx* ctx, float* x, float* v, float* rho, float* lambda) {
  if (!ctx) return PBF_ERR_ARG;
  if (ctx->n == 0) return PBF_OK;
  const size_t n = ctx->n;
  float* sx = ctx->stage;
  float* sv = ctx->stage + 3 * ctx->capacity;
  int rc;
  if (x) {
    if ((rc = get_array_dev(ctx, PBF_ARRAY_POSITIONS, sx))) return rc;
    CK(cudaMemcpyAsync(x, sx, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (v) {
    if ((rc = get_array_dev(ctx, PBF_ARRAY_VELOCITIES, sv))) return rc;
    CK(cudaMemcpyAsync(v, sv, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (rho || lambda) {
    CK(cudaStreamSynchronize(ctx->stream));
    if (rho) {
      if ((rc = get_array_dev(ctx, PBF_ARRAY_DENSITIES, sx))) return rc;
      CK(cudaMemcpyAsync(rho, sx, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (lambda) {
      if ((rc = get_array_dev(ctx, PBF_ARRAY_LAMBDAS, sv))) return rc;
      CK(cudaMemcpyAsync(lambda, sv, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

// ---- stages ----
#define STAGE_PROLOGUE(b, e)              \
  if (!ctx) return PBF_ERR_ARG;           \
  {                                       \
    int rc_ = check_span(ctx, b, e);      \
    if (rc_) return rc_;                  \
  }                                       \
  if (ctx->n == 0) return PBF_OK;         \
  const int n = (int)ctx->n;              \
  const int g = blocks_for(ctx->n);       \
  (void)g;                                \
  const bool X = ctx->params.exact_math != 0; \
  (void)X;                                \
  const Dev SP = span_dev(ctx, e);        \
  (void)SP;

int pbf_apply_external_forces(pbf_ctx* ctx, size_t b, size_t e) {
  STAGE_PROLOGUE(b, e);
  k_external<<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->velH);
  return check_launch(ctx, "apply_external_forces");
}

int pbf_predict_positions(pbf_ctx* ctx, size_t b, size_t e) {
  STAGE_PROLOGUE(b, e);
  k_predict<<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->posH, ctx->velH, ctx->pstH);
  return check_launch(ctx, "predict_positions");
}

int pbf_find_neighbors(pbf_ctx* ctx, size_t bin_b, size_t bin_e, size_t fill_b, size_t fill_e) {
  if (!ctx) return PBF_ERR_ARG;
  int rc = check_span(ctx, bin_b, bin_e);
  if (rc) return rc;
  if ((rc = check_span(ctx, fill_b, fill_e))) return rc;
  if (bin_e != ctx->n)
    return fail(ctx, PBF_ERR_SPAN, "find_neighbors bins every held particle: bin span [0, %zu) given, [0, %zu) held",
                bin_e, ctx->n);
  if (ctx->n == 0) {
    ctx->lists_valid = true;
    return PBF_OK;
  }
  const int n = (int)ctx->n, g = blocks_for(ctx->n);
  cudaStream_t s = ctx->stream;
  CK(cudaMemsetAsync(ctx->cell_count, 0, sizeof(uint32_t) * ((size_t)ctx->nbins + 1), s));  // + the crowded flag
  k_hash<<<g, kBlock, 0, s>>>(ctx->dev, n, ctx->pstH, ctx->origH, ctx->key, ctx->cell_count, ctx->key_ref,
                              ctx->pairs, ctx->err);
  launch_sort_to_pairs(ctx);
  k_reorder<true><<<g, kBlock, 0, s>>>(n, ctx->sorted, ctx->key, ctx->posH, ctx->pstH, ctx->velH, ctx->scrH,
                                       ctx->lamH, ctx->posS, ctx->pstS, ctx->velS, ctx->scrS, ctx->lamS, ctx->origS,
                                       ctx->keyH);
  const size_t f4 = sizeof(float4) * ctx->n;
  CK(cudaMemcpyAsync(ctx->posH, ctx->posS, f4, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(ctx->pstH, ctx->pstS, f4, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(ctx->velH, ctx->velS, f4, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(ctx->scrH, ctx->scrS, f4, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(ctx->lamH, ctx->lamS, sizeof(float) * ctx->n, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(ctx->origH, ctx->origS, sizeof(uint32_t) * ctx->n, cudaMemcpyDeviceToDevice, s));
  launch_fill(ctx, ctx->pstH);
  if (fill_e < ctx->n)  // particles outside the fill span (halo particles) get empty lists
    k_clear_outside_span<<<g, kBlock, 0, s>>>(n, ctx->origH, (uint32_t)fill_e, ctx->cnt);
  rc = check_launch(ctx, "find_neighbors");
  if (rc) return rc;
  ctx->lists_valid = true;
  return PBF_OK;
}

int pbf_compute_densities(pbf_ctx* ctx, size_t b, size_t e) {
  STAGE_PROLOGUE(b, e);
  if (int rc = need_lists(ctx)) return rc;
  if (X) k_density<true><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->velH, ctx->pstS);
  else k_density<false><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->velH, ctx->pstS);
  CK(cudaMemcpyAsync(ctx->pstH, ctx->pstS, sizeof(float4) * ctx->n, cudaMemcpyDeviceToDevice, ctx->stream));
  return check_launch(ctx, "compute_densities");
}

int pbf_compute_pressure_lambdas(pbf_ctx* ctx, size_t b, size_t e) {
  STAGE_PROLOGUE(b, e);
  if (int rc = need_lists(ctx)) return rc;
  if (X) k_lambda<true><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->velH, ctx->lamH);
  else k_lambda<false><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->velH, ctx->lamH);
  return check_launch(ctx, "compute_pressure_lambdas");
}

int pbf_compute_pressure_dps(pbf_ctx* ctx, size_t b, size_t e, int substep) {
  (void)substep;  // unused by the reference too (particles.h:348)
  STAGE_PROLOGUE(b, e);
  if (int rc = need_lists(ctx)) return rc;
  const bool SC = ctx->params.scorr_k > 0.0f;
  const Dev& P = SP;
  if (X && SC) k_dp<true, true><<<g, kBlock, 0, ctx->stream>>>(P, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->lamH, ctx->scrH);
  else if (X) k_dp<true, false><<<g, kBlock, 0, ctx->stream>>>(P, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->lamH, ctx->scrH);
  else if (SC) k_dp<false, true><<<g, kBlock, 0, ctx->stream>>>(P, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->lamH, ctx->scrH);
  else k_dp<false, false><<<g, kBlock, 0, ctx->stream>>>(P, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->lamH, ctx->scrH);
  return check_launch(ctx, "compute_pressure_dps");
}

int pbf_update_position_stars(pbf_ctx* ctx, size_t b, size_t e) {
  STAGE_PROLOGUE(b, e);
  k_update_xs<<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->pstH, ctx->scrH);
  return check_launch(ctx, "update_position_stars");
}

int pbf_update_velocities(pbf_ctx* ctx, size_t b, size_t e) {
  STAGE_PROLOGUE(b, e);
  k_update_v<<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->pstH, ctx->posH, ctx->velH);
  return check_launch(ctx, "update_velocities");
}

int pbf_apply_surface_tension(pbf_ctx* ctx, size_t cb, size_t ce, size_t sb, size_t se) {
  if (!ctx) return PBF_ERR_ARG;
  if (int rc = check_span(ctx, sb, se)) return rc;
  STAGE_PROLOGUE(cb, ce);
  if (int rc = need_lists(ctx)) return rc;
  if (X) k_color<true><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->velH, ctx->scrH);
  else k_color<false><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->velH, ctx->scrH);
  k_surface<<<g, kBlock, 0, ctx->stream>>>(span_dev(ctx, se), n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->scrH, ctx->velH);
  return check_launch(ctx, "apply_surface_tension");
}

int pbf_apply_viscosity(pbf_ctx* ctx, size_t b, size_t e) {
  STAGE_PROLOGUE(b, e);
  if (int rc = need_lists(ctx)) return rc;
  if (X) k_viscosity<true, false><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->velH, ctx->velT, nullptr, nullptr, nullptr, nullptr);
  else k_viscosity<false, false><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->velH, ctx->velT, nullptr, nullptr, nullptr, nullptr);
  CK(cudaMemcpyAsync(ctx->velH, ctx->velT, sizeof(float4) * ctx->n, cudaMemcpyDeviceToDevice, ctx->stream));
  return check_launch(ctx, "apply_viscosity");
}

int pbf_compute_vorticity(pbf_ctx* ctx, size_t b, size_t e) {
  STAGE_PROLOGUE(b, e);
  if (int rc = need_lists(ctx)) return rc;
  if (X) k_vorticity<true><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->velH, ctx->scrH, nullptr);
  else k_vorticity<false><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, ctx->pstH, ctx->velH, ctx->scrH, nullptr);
  return check_launch(ctx, "compute_vorticity");
}

int pbf_apply_vorticity(pbf_ctx* ctx, size_t b, size_t e) {
  STAGE_PROLOGUE(b, e);
  if (int rc = need_lists(ctx)) return rc;
  if (X) k_apply_vorticity<true, false><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, nullptr, ctx->pstH, ctx->scrH, ctx->velH);
  else k_apply_vorticity<false, false><<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->lstride, ctx->nbr, ctx->cnt, nullptr, ctx->pstH, ctx->scrH, ctx->velH);
  return check_launch(ctx, "apply_vorticity");
}

int pbf_update_positions(pbf_ctx* ctx, size_t b, size_t e) {
  STAGE_PROLOGUE(b, e);
  if (e == ctx->n) {
    CK(cudaMemcpyAsync(ctx->posH, ctx->pstH, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
    return PBF_OK;
  }
  k_update_positions<<<g, kBlock, 0, ctx->stream>>>(SP, n, ctx->pstH, ctx->posH);
  return check_launch(ctx, "update_positions");
}

// nsteps fused steps captured from the context's stream into a graph (not
// instantiated; the caller owns it).
static int capture_steps(pbf_ctx* ctx, int nsteps, cudaGraph_t* out) {
  cudaGraph_t graph = nullptr;
  ctx->capture_failed = false;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < nsteps; ++i) launch_step(ctx);
  cudaError_t le = cudaGetLastError();
  cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
  if (le != cudaSuccess || ce != cudaSuccess || ctx->capture_failed) {
    if (graph) cudaGraphDestroy(graph);
    const bool loop = ctx->capture_failed;
    ctx->capture_failed = false;
    if (loop) return fail(ctx, PBF_ERR_CUDA, "graph capture of the learned solver's iteration loop failed");
    return fail(ctx, PBF_ERR_CUDA, "graph capture failed: %s / %s", cudaGetErrorString(le), cudaGetErrorString(ce));
  }
  *out = graph;
  return PBF_OK;
}

int pbf_step(pbf_ctx* ctx, int nsteps) {
  if (!ctx || nsteps < 0) return PBF_ERR_ARG;
  if (nsteps == 0) return PBF_OK;
  if (ctx->params.solver == 1 && !ctx->mlp_ready)
    return fail(ctx, PBF_ERR_STATE, "learned solver without a network: call pbf_mlp_init or pbf_mlp_set");
  if (ctx->n == 0) {
    ctx->lists_valid = true;  // an empty set has (empty) lists
    return PBF_OK;
  }
  ctx->steps_done += (uint64_t)nsteps;
  if (ctx->timing) {
    for (int i = 0; i < nsteps; ++i) launch_step(ctx);
    int rc = check_launch(ctx, "step");
    if (rc) return rc;
    ctx->lists_valid = true;
    return harvest_times(ctx);
  }
  auto it = ctx->graphs.find(nsteps);
  if (it == ctx->graphs.end()) {
    cudaGraph_t graph = nullptr;
    if (int rc = capture_steps(ctx, nsteps, &graph)) return rc;
    cudaGraphExec_t exec = nullptr;
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return fail(ctx, PBF_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ie));
    it = ctx->graphs.emplace(nsteps, exec).first;
  }
  CK(cudaGraphLaunch(it->second, ctx->stream));
  ctx->lists_valid = true;
  return PBF_OK;
}

// ---- scene groups: independent contexts advanced by one graph launch ----
// The group's graph holds, per member context, its nsteps-step chain as a
// child graph, with no edge between members: one launch, and every scene
// advances at its own pace (a light scene's steps run while a crowded one is
// in its list fill), where the one-context batch ends every step when its
// slowest scene ends.  Results are each context's own pbf_step results, bit
// for bit.  The graph is cached per nsteps and rebuilt when a member drops its
// graphs (a new particle count or new parameters).
constexpr bool kGroupPriorities = true;  // members' kernels prioritised by scene size

struct pbf_group {
  std::vector<pbf_ctx*> ctxs;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  std::vector<cudaEvent_t> ready;
  struct Built {
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> epochs;
  };
  std::map<int, Built> graphs;
};

static void group_drop(pbf_group* g) {
  for (auto& kv : g->graphs) cudaGraphExecDestroy(kv.second.exec);
  g->graphs.clear();
}

int pbf_group_create(pbf_ctx* const* ctxs, int n, pbf_group** out) {
  if (!out || !ctxs || n < 1) return fail(nullptr, PBF_ERR_ARG, "pbf_group_create: no contexts");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i]) return fail(nullptr, PBF_ERR_ARG, "pbf_group_create: context %d is NULL", i);
    for (int j = 0; j < i; ++j)
      if (ctxs[j] == ctxs[i]) return fail(nullptr, PBF_ERR_ARG, "pbf_group_create: context %d listed twice", i);
  }
  auto* g = new pbf_group();
  g->ctxs.assign(ctxs, ctxs + n);
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming);
  g->ready.assign((size_t)n, nullptr);
  for (int i = 0; i < n && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&g->ready[i], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    pbf_group_destroy(g);
    return fail(nullptr, PBF_ERR_CUDA, "pbf_group_create: %s", cudaGetErrorString(e));
  }
  *out = g;
  return PBF_OK;
}

int pbf_group_step(pbf_group* g, int nsteps) {
  if (!g || nsteps < 0) return fail(nullptr, PBF_ERR_ARG, "pbf_group_step: bad arguments");
  if (nsteps == 0) return PBF_OK;
  for (pbf_ctx* c : g->ctxs) {
    if (c->timing) return fail(nullptr, PBF_ERR_STATE, "pbf_group_step: a member has per-kernel timing on");
    if (c->params.solver == 1 && !c->mlp_ready)
      return fail(nullptr, PBF_ERR_STATE, "pbf_group_step: a learned-solver member has no network");
  }
  auto it = g->graphs.find(nsteps);
  if (it != g->graphs.end()) {
    bool stale = false;
    for (size_t i = 0; i < g->ctxs.size(); ++i) stale = stale || it->second.epochs[i] != g->ctxs[i]->graph_epoch;
    if (stale) {
      cudaGraphExecDestroy(it->second.exec);
      g->graphs.erase(it);
      it = g->graphs.end();
    }
  }
  if (it == g->graphs.end()) {
    cudaGraph_t parent = nullptr;
    if (cudaGraphCreate(&parent, 0) != cudaSuccess) return fail(nullptr, PBF_ERR_CUDA, "pbf_group_step: graph");
    pbf_group::Built b;
    for (pbf_ctx* c : g->ctxs) b.epochs.push_back(c->graph_epoch);
    // members in descending particle count: the largest scenes' chains enter
    // the graph first, and their kernels run at the higher stream priorities
    // (the graph is instantiated with node priorities), so the longest chains
    // start first and the small scenes fill the GPU around them
    std::vector<pbf_ctx*> order(g->ctxs);
    std::stable_sort(order.begin(), order.end(), [](const pbf_ctx* a, const pbf_ctx* b) { return a->n > b->n; });
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    const int levels = least - greatest + 1;  // e.g. 0 (lowest) .. -5 (highest)
    for (size_t rank = 0; rank < order.size(); ++rank) {
      pbf_ctx* c = order[rank];
      if (c->n == 0) continue;
      cudaGraph_t child = nullptr;
      if (int rc = capture_steps(c, nsteps, &child)) {
        cudaGraphDestroy(parent);
        return fail(nullptr, rc, "pbf_group_step: capture of a member failed: %s", pbf_last_error(c));
      }
      if (kGroupPriorities && levels > 1) {
        const int prio = greatest + (int)((rank * (size_t)levels) / order.size());
        size_t nn = 0;
        cudaGraphGetNodes(child, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        if (nn && cudaGraphGetNodes(child, nodes.data(), &nn) == cudaSuccess) {
          cudaLaunchAttributeValue v = {};
          v.priority = prio;
          for (cudaGraphNode_t node : nodes) {
            cudaGraphNodeType type;
            if (cudaGraphNodeGetType(node, &type) == cudaSuccess && type == cudaGraphNodeTypeKernel)
              cudaGraphKernelNodeSetAttribute(node, cudaLaunchAttributePriority, &v);
          }
        }
        cudaGetLastError();  // a priority that does not apply leaves the default
      }
      cudaGraphNode_t node = nullptr;
      const cudaError_t e = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, child);
      cudaGraphDestroy(child);  // the node holds its own copy
      if (e != cudaSuccess) {
        cudaGraphDestroy(parent);
        return fail(nullptr, PBF_ERR_CUDA, "pbf_group_step: a member's steps cannot be a child graph (%s)",
                    cudaGetErrorString(e));
      }
    }
    const cudaError_t ie =
        cudaGraphInstantiate(&b.exec, parent, kGroupPriorities ? cudaGraphInstantiateFlagUseNodePriority : 0);
    cudaGraphDestroy(parent);
    if (ie != cudaSuccess)
      return fail(nullptr, PBF_ERR_CUDA, "pbf_group_step: graph instantiate failed: %s", cudaGetErrorString(ie));
    it = g->graphs.emplace(nsteps, b).first;
  }
  // the launch follows each member's pending work, and each member's next work follows the launch
  cudaError_t e = cudaSuccess;
  for (size_t i = 0; i < g->ctxs.size() && e == cudaSuccess; ++i) {
    e = cudaEventRecord(g->ready[i], g->ctxs[i]->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(g->stream, g->ready[i], 0);
  }
  if (e == cudaSuccess) e = cudaGraphLaunch(it->second.exec, g->stream);
  if (e == cudaSuccess) e = cudaEventRecord(g->done, g->stream);
  for (size_t i = 0; i < g->ctxs.size() && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(g->ctxs[i]->stream, g->done, 0);
  if (e != cudaSuccess) return fail(nullptr, PBF_ERR_CUDA, "pbf_group_step: launch: %s", cudaGetErrorString(e));
  for (pbf_ctx* c : g->ctxs) {
    if (c->n == 0) continue;
    c->steps_done += (uint64_t)nsteps;
    c->lists_valid = true;
  }
  return PBF_OK;
}

int pbf_group_sync(pbf_group* g) {
  if (!g) return PBF_ERR_ARG;
  const cudaError_t e = cudaStreamSynchronize(g->stream);
  return e == cudaSuccess ? PBF_OK : fail(nullptr, PBF_ERR_CUDA, "pbf_group_sync: %s", cudaGetErrorString(e));
}

int pbf_group_get_stream(pbf_group* g, void** stream_out) {
  if (!g || !stream_out) return PBF_ERR_ARG;
  *stream_out = g->stream;
  return PBF_OK;
}

void pbf_group_destroy(pbf_group* g) {
  if (!g) return;
  if (g->stream) cudaStreamSynchronize(g->stream);
  group_drop(g);
  for (cudaEvent_t e : g->ready)
    if (e) cudaEventDestroy(e);
  if (g->done) cudaEventDestroy(g->done);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

int pbf_sync(pbf_ctx* ctx) {
  if (!ctx) return PBF_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

int pbf_get_stream(pbf_ctx* ctx, void** stream_out) {
  if (!ctx || !stream_out) return PBF_ERR_ARG;
  *stream_out = (void*)ctx->stream;
  return PBF_OK;
}

int pbf_get_neighbors(pbf_ctx* ctx, int32_t* idx, int32_t* count) {
  if (!ctx) return PBF_ERR_ARG;
  if (int rc = need_lists(ctx)) return rc;
  if (ctx->n == 0) return PBF_OK;
  const size_t n = ctx->n, cap = (size_t)ctx->params.neighbor_cap;
  int32_t* di = ctx->stage_i;
  int32_t* dc = ctx->stage_i + n * cap;
  k_export_neighbors<<<blocks_for(n), kBlock, 0, ctx->stream>>>((int)n, ctx->lstride, (int)cap, ctx->nbr, ctx->cnt,
                                                                 ctx->origH, di, dc,
                                                                 ctx->lists_slot_order ? ctx->seg : nullptr,
                                                                 ctx->fill_words + kFillLastOrder);
  if (int rc = check_launch(ctx, "export_neighbors")) return rc;
  if (idx) CK(cudaMemcpyAsync(idx, di, n * cap * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  if (count) CK(cudaMemcpyAsync(count, dc, n * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

int pbf_get_bins(pbf_ctx* ctx, uint32_t* sorted_keys, uint32_t* sorted_ids, uint32_t* bin_begin,
                 uint32_t* bin_end) {
  if (!ctx) return PBF_ERR_ARG;
  if (int rc = need_lists(ctx)) return rc;
  const size_t n = ctx->n, B = (size_t)ctx->nbins;
  if (sorted_keys && n) CK(cudaMemcpyAsync(sorted_keys, ctx->keyH, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (sorted_ids && n) CK(cudaMemcpyAsync(sorted_ids, ctx->origH, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (bin_begin) CK(cudaMemcpyAsync(bin_begin, ctx->cell_start, B * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (bin_end) CK(cudaMemcpyAsync(bin_end, ctx->cell_start + 1, B * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

// Statistics over the particles in slots [b0, b1) (one scene of a batch, or
// all); the error flags are read, and cleared when `clear_flags`.
static int stats_range(pbf_ctx* ctx, size_t b0, size_t b1, bool clear_flags, pbf_stats_t* out) {
  std::memset(out, 0, sizeof(*out));
  out->n = b1 - b0;
  if (int rc = need_lists(ctx)) return rc;
  cudaStream_t s = ctx->stream;
  CK(cudaMemsetAsync(ctx->acc, 0, 8 * sizeof(double), s));
  CK(cudaMemsetAsync(ctx->maxerr, 0, sizeof(unsigned long long), s));
  CK(cudaMemsetAsync(ctx->hits, 0, sizeof(unsigned long long), s));
  if (b1 > b0) {
    k_stats<<<blocks_for(b1 - b0), kBlock, 0, s>>>(ctx->dev, (int)b0, (int)b1, ctx->lstride, ctx->nbr, ctx->cnt,
                                                   ctx->pstH, ctx->posH, ctx->velH, ctx->acc, ctx->maxerr,
                                                   ctx->hits);
    if (int rc = check_launch(ctx, "stats")) return rc;
  }
  double acc[8];
  unsigned long long mx = 0, hits = 0;
  uint32_t err = 0;
  CK(cudaMemcpyAsync(acc, ctx->acc, sizeof(acc), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&mx, ctx->maxerr, sizeof(mx), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&hits, ctx->hits, sizeof(hits), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&err, ctx->err, sizeof(err), cudaMemcpyDeviceToHost, s));
  if (clear_flags) CK(cudaMemsetAsync(ctx->err, 0, sizeof(uint32_t), s));
  CK(cudaStreamSynchronize(s));
  const double n = b1 > b0 ? (double)(b1 - b0) : 1.0;
  double maxerr;
  std::memcpy(&maxerr, &mx, sizeof(double));
  out->mean_density_error = acc[0] / n;
  out->max_density_error = maxerr;
  out->kinetic_energy = acc[1];
  out->center_of_mass[0] = acc[2] / n;
  out->center_of_mass[1] = acc[3] / n;
  out->center_of_mass[2] = acc[4] / n;
  out->mean_neighbors = acc[5] / n;
  out->cap_hits = hits;
  out->error_flags = err;
  if (ctx->params.solver == 1 && !(ctx->params.residual_tol > 0.0f)) {  // a fixed count, no checks
    out->solver_iterations = (uint32_t)std::max(ctx->params.max_iterations, 1);
    out->solver_residual = -1.0;
  } else if (ctx->params.solver == 1) {
    pbf::SolveState stt;
    CK(cudaMemcpy(&stt, ctx->state, sizeof(stt), cudaMemcpyDeviceToHost));
    out->solver_iterations = 1u + stt.iterations;
    out->solver_residual = stt.residual;
  } else {
    out->solver_iterations = (uint32_t)ctx->params.solve_steps;
    out->solver_residual = -1.0;
  }
  if (!ctx->params.exact_math) CK(cudaMemcpy(&out->lists_slot_order, ctx->fill_words + kFillLastOrder,
                                             sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (any_staged(ctx) && ctx->n) {  // the tiles of the last list fill
    const size_t tiles = (ctx->n + kTile - 1) / kTile;
    std::vector<int32_t> nr(tiles);
    CK(cudaMemcpy(nr.data(), ctx->tile_nruns, tiles * sizeof(int32_t), cudaMemcpyDeviceToHost));
    out->tiles = (uint32_t)tiles;
    for (int32_t v : nr) out->tiles_staged += v > 0 ? 1u : 0u;
  }
  return PBF_OK;
}

int pbf_stats(pbf_ctx* ctx, pbf_stats_t* out) {
  if (!ctx || !out) return PBF_ERR_ARG;
  return stats_range(ctx, 0, ctx->n, true, out);
}

int pbf_scene_count(const pbf_ctx* ctx) { return ctx ? (int)ctx->scenes.size() : 0; }

int pbf_scene_stats(pbf_ctx* ctx, int scene, pbf_stats_t* out) {
  if (!ctx || !out) return PBF_ERR_ARG;
  if (ctx->scenes.empty()) {
    if (scene != 0) return fail(ctx, PBF_ERR_ARG, "scene %d of a single-scene context", scene);
    return stats_range(ctx, 0, ctx->n, false, out);
  }
  if (scene < 0 || scene >= (int)ctx->scenes.size())
    return fail(ctx, PBF_ERR_ARG, "scene %d out of [0, %zu)", scene, ctx->scenes.size());
  if (ctx->n == 0) return stats_range(ctx, 0, 0, false, out);
  return stats_range(ctx, ctx->scene_first[scene], ctx->scene_first[scene + 1], false, out);
}

// ---- learned warm start ----
static int mlp_refresh(pbf_ctx* ctx) {
  pbf::k_mlp_sync<<<(pbf::kMlpH * pbf::kMlpH + 255) / 256, 256, 0, ctx->stream>>>(ctx->mlp_params, ctx->w1b, ctx->w2b,
                                                                                ctx->w2tb);
  return check_launch(ctx, "mlp_sync");
}

int pbf_mlp_init(pbf_ctx* ctx, uint64_t seed) {
  if (!ctx) return PBF_ERR_ARG;
  // Xavier-uniform weights from a SplitMix64 stream, zero biases.
  std::vector<float> P(pbf::kMlpParams, 0.0f);
  uint64_t z = seed;
  auto uni = [&]() {
    z += 0x9E3779B97F4A7C15ull;
    uint64_t r = z;
    r = (r ^ (r >> 30)) * 0xBF58476D1CE4E5B9ull;
    r = (r ^ (r >> 27)) * 0x94D049BB133111EBull;
    r ^= r >> 31;
    return (float)(r >> 40) * 0x1p-24f * 2.0f - 1.0f;
  };
  const float a1 = std::sqrt(6.0f / (pbf::kMlpIn + pbf::kMlpH)), a2 = std::sqrt(6.0f / (2 * pbf::kMlpH)),
              a3 = std::sqrt(6.0f / (pbf::kMlpH + 1));
  for (int i = 0; i < pbf::kMlpH * pbf::kMlpIn; ++i) P[pbf::kOffW1 + i] = a1 * uni();
  for (int i = 0; i < pbf::kMlpH * pbf::kMlpH; ++i) P[pbf::kOffW2 + i] = a2 * uni();
  for (int i = 0; i < pbf::kMlpH; ++i) P[pbf::kOffW3 + i] = a3 * uni();
  std::vector<float> norm(PBF_MLP_NORM, 0.0f);
  for (int k = 0; k < pbf::kMlpIn; ++k) norm[pbf::kMlpIn + k] = 1.0f;
  norm[2 * pbf::kMlpIn] = 1.0f;
  return pbf_mlp_set(ctx, P.data(), norm.data());
}

int pbf_mlp_set(pbf_ctx* ctx, const float* params, const float* norm) {
  if (!ctx || !params || !norm) return PBF_ERR_ARG;
  if (!(norm[2 * pbf::kMlpIn] != 0.0f)) return fail(ctx, PBF_ERR_ARG, "label_scale must be nonzero");
  CK(cudaMemcpyAsync(ctx->mlp_params, params, sizeof(float) * pbf::kMlpParams, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->mlp_norm, norm, sizeof(float) * PBF_MLP_NORM, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ctx->mlp_m, 0, sizeof(float) * pbf::kMlpParams, ctx->stream));
  CK(cudaMemsetAsync(ctx->mlp_v, 0, sizeof(float) * pbf::kMlpParams, ctx->stream));
  ctx->label_scale = norm[2 * pbf::kMlpIn];
  ctx->adam_t = 0;
  if (int rc = mlp_refresh(ctx)) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->mlp_ready = true;
  drop_graphs(ctx);  // the label scale is a kernel argument of the learned step
  return PBF_OK;
}

int pbf_mlp_get(pbf_ctx* ctx, float* params, float* norm) {
  if (!ctx) return PBF_ERR_ARG;
  if (params)
    CK(cudaMemcpyAsync(params, ctx->mlp_params, sizeof(float) * pbf::kMlpParams, cudaMemcpyDeviceToHost, ctx->stream));
  if (norm) CK(cudaMemcpyAsync(norm, ctx->mlp_norm, sizeof(float) * PBF_MLP_NORM, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

int pbf_set_recording(pbf_ctx* ctx, int on) {
  if (!ctx) return PBF_ERR_ARG;
  if (on && !ctx->feats) {
    if (int rc = dalloc(ctx, &ctx->feats, ctx->capacity * pbf::kMlpIn)) return rc;
    CK(cudaMemsetAsync(ctx->feats, 0, ctx->capacity * pbf::kMlpIn * sizeof(float), ctx->stream));
  }
  if ((on != 0) != ctx->recording) drop_graphs(ctx);
  ctx->recording = on != 0;
  return PBF_OK;
}

int pbf_get_training_data(pbf_ctx* ctx, float* features, float* labels) {
  if (!ctx) return PBF_ERR_ARG;
  if (!ctx->feats) return fail(ctx, PBF_ERR_STATE, "no recorded step: call pbf_set_recording(ctx, 1) and step");
  const size_t n = ctx->n;
  if (features && n)
    CK(cudaMemcpyAsync(features, ctx->feats, n * pbf::kMlpIn * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  if (labels && n) CK(cudaMemcpyAsync(labels, ctx->lamsumH, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

// The tensor-core training kernel: one CTA per SM (its 138 KB of operands),
// at most one per 128-sample tile.
static int grad_tc_setup(pbf_ctx* ctx) {
  const cudaError_t e1 = cudaFuncSetAttribute(pbf::k_mlp_grad_tc<true, true>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, pbf::tt::kSmemBytes);
  const cudaError_t e2 = cudaFuncSetAttribute(pbf::k_mlp_grad_tc<false, false>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, pbf::tt::kSmemBytes);
  if (e1 != cudaSuccess || e2 != cudaSuccess)
    return fail(ctx, PBF_ERR_CUDA, "training kernel shared memory: %s", cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
  return PBF_OK;
}

static int grad_tc_grid(const pbf_ctx* ctx, int batch) {
  const int tiles = (batch + pbf::tc::kRows - 1) / pbf::tc::kRows;
  return std::max(1, std::min(ctx->sms, tiles));
}

int pbf_mlp_train(pbf_ctx* ctx, int adam_steps, int batch, float lr, uint64_t seed, float* loss) {
  if (!ctx || adam_steps < 0 || batch < 1) return PBF_ERR_ARG;
  if (!ctx->mlp_ready) return fail(ctx, PBF_ERR_STATE, "no network: call pbf_mlp_init or pbf_mlp_set");
  if (!ctx->feats || ctx->n == 0) return fail(ctx, PBF_ERR_STATE, "no recorded step to train on");
  const pbf::MlpDev M = mlp_dev(ctx);
  if (int rc = grad_tc_setup(ctx)) return rc;
  for (int it = 0; it < adam_steps; ++it) {
    CK(cudaMemsetAsync(ctx->mlp_grad, 0, sizeof(float) * pbf::kMlpParams, ctx->stream));
    CK(cudaMemsetAsync(ctx->mlp_loss, 0, sizeof(float), ctx->stream));
    pbf::k_mlp_grad_tc<true, true><<<grad_tc_grid(ctx, batch), pbf::tc::kThreads, pbf::tt::kSmemBytes,
                                      ctx->stream>>>(M, ctx->feats, ctx->lamsumH, (int)ctx->n, batch,
                                                     seed + 0x632BE59BD9B4E019ull * (uint64_t)it,
                                                     1.0f / ctx->label_scale, ctx->mlp_grad, ctx->mlp_loss,
                                                     ctx->err);
    ctx->adam_t += 1;
    const float c1 = 1.0f / (1.0f - std::pow(0.9f, (float)ctx->adam_t));
    const float c2 = 1.0f / (1.0f - std::pow(0.999f, (float)ctx->adam_t));
    pbf::k_mlp_adam<<<(pbf::kMlpParams + 255) / 256, 256, 0, ctx->stream>>>(ctx->mlp_params, ctx->mlp_grad, ctx->mlp_m,
                                                                           ctx->mlp_v, pbf::kMlpParams, lr, c1, c2);
    if (int rc = mlp_refresh(ctx)) return rc;
  }
  if (int rc = check_launch(ctx, "mlp_train")) return rc;
  if (loss) CK(cudaMemcpyAsync(loss, ctx->mlp_loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

int pbf_mlp_gradients(pbf_ctx* ctx, const float* features, const float* targets, size_t n, float* grad,
                      float* loss) {
  if (!ctx || !features || !targets || n == 0) return PBF_ERR_ARG;
  if (n * (pbf::kMlpIn + 1) > 6 * ctx->capacity)
    return fail(ctx, PBF_ERR_CAPACITY, "%zu samples exceed the staging area of this context", n);
  if (!ctx->mlp_ready) return fail(ctx, PBF_ERR_STATE, "no network: call pbf_mlp_init or pbf_mlp_set");
  float* df = ctx->stage;
  float* dt = ctx->stage + n * pbf::kMlpIn;
  CK(cudaMemcpyAsync(df, features, n * pbf::kMlpIn * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dt, targets, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ctx->mlp_grad, 0, sizeof(float) * pbf::kMlpParams, ctx->stream));
  CK(cudaMemsetAsync(ctx->mlp_loss, 0, sizeof(float), ctx->stream));
  if (int rc = grad_tc_setup(ctx)) return rc;
  pbf::k_mlp_grad_tc<false, false><<<grad_tc_grid(ctx, (int)n), pbf::tc::kThreads, pbf::tt::kSmemBytes,
                                     ctx->stream>>>(mlp_dev(ctx), df, dt, (int)n, (int)n, 0, 1.0f, ctx->mlp_grad,
                                                    ctx->mlp_loss, ctx->err);
  if (int rc = check_launch(ctx, "mlp_gradients")) return rc;
  if (grad)
    CK(cudaMemcpyAsync(grad, ctx->mlp_grad, sizeof(float) * pbf::kMlpParams, cudaMemcpyDeviceToHost, ctx->stream));
  if (loss) CK(cudaMemcpyAsync(loss, ctx->mlp_loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

int pbf_mlp_predict(pbf_ctx* ctx, const float* features, size_t n, float* y) {
  if (!ctx || !features || !y || n == 0) return PBF_ERR_ARG;
  if (n * (pbf::kMlpIn + 1) > 6 * ctx->capacity)
    return fail(ctx, PBF_ERR_CAPACITY, "%zu samples exceed the staging area of this context", n);
  if (!ctx->mlp_ready) return fail(ctx, PBF_ERR_STATE, "no network: call pbf_mlp_init or pbf_mlp_set");
  float* df = ctx->stage;
  float* dy = ctx->stage + n * pbf::kMlpIn;
  CK(cudaMemcpyAsync(df, features, n * pbf::kMlpIn * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  kl_mlp_tc<false><<<mlp_tc_grid(ctx, (int)n), pbf::tc::kThreads, 0, ctx->stream>>>(
      mlp_dev(ctx), (int)n, nullptr, df, nullptr, nullptr, nullptr, dy, ctx->err);
  if (int rc = check_launch(ctx, "mlp_predict")) return rc;
  uint32_t err = 0;
  CK(cudaMemcpyAsync(y, dy, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&err, ctx->err, sizeof(err), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  // the context's error word (the step's flags are kept: a timeout raised by
  // an earlier step fails this call too, the context's tensor-core path has failed)
  if (err & PBF_FLAG_WAIT_TIMEOUT) return fail(ctx, PBF_ERR_DEVICE, "mlp_predict: a tensor-core wait timed out");
  return PBF_OK;
}

int pbf_selftest_mlp_wait_timeout(pbf_ctx* ctx, uint32_t* flags) {
  if (!ctx || !flags) return PBF_ERR_ARG;
  if (!ctx->mlp_ready) return fail(ctx, PBF_ERR_STATE, "no network: call pbf_mlp_init or pbf_mlp_set");
  const int rows = pbf::tc::kRows;  // one tile, one CTA
  const size_t need = (size_t)rows * (pbf::kMlpIn + 1) + 1;
  if (need > 6 * ctx->capacity)
    return fail(ctx, PBF_ERR_CAPACITY, "the self-test needs a context of at least %zu particles", need / 6 + 1);
  float* df = ctx->stage;
  float* dy = ctx->stage + (size_t)rows * pbf::kMlpIn;
  uint32_t* status = reinterpret_cast<uint32_t*>(dy + rows);
  CK(cudaMemsetAsync(ctx->stage, 0, need * sizeof(float), ctx->stream));
  kl_mlp_tc<false, true><<<1, pbf::tc::kThreads, 0, ctx->stream>>>(mlp_dev(ctx), rows, nullptr, df, nullptr, nullptr,
                                                                   nullptr, dy, status);
  if (int rc = check_launch(ctx, "selftest_mlp_wait_timeout")) return rc;
  CK(cudaMemcpyAsync(flags, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

int pbf_set_persistent(pbf_ctx* ctx, int enable) {
  if (!ctx) return PBF_ERR_ARG;
  if (!enable) {
    if (ctx->persistent) drop_graphs(ctx);
    ctx->persistent = false;
    return PBF_OK;
  }
  if (ctx->scenes.empty())
    return fail(ctx, PBF_ERR_STATE, "the persistent step runs batches of scenes (pbf_create_batch)");
  if (!persist_supported(ctx))
    return fail(ctx, PBF_ERR_PARAMS, "the persistent step runs fast math, the plain solver with 1..%d iterations, "
                                     "no surface tension and no s_corr", kPersistMaxK);
  if (!ctx->persist_words) {
    int rc;
    if ((rc = dalloc(ctx, &ctx->persist_words, 2)) ||
        (rc = dalloc(ctx, &ctx->persist_done, (size_t)kPersistMaxPasses * ctx->scenes.size())))
      return rc;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persist<false>, kPersistThreads, 0) != cudaSuccess ||
        per_sm <= 0)
      per_sm = 1;
    ctx->persist_grid = ctx->sms * per_sm;
  }
  if (!ctx->persistent) drop_graphs(ctx);
  ctx->persistent = true;
  return PBF_OK;
}

int pbf_selftest_persistent_wait_timeout(pbf_ctx* ctx, uint32_t* flags) {
  if (!ctx || !flags) return PBF_ERR_ARG;
  if (6 * ctx->capacity < 8)
    return fail(ctx, PBF_ERR_CAPACITY, "the self-test needs a context of at least 2 particles");
  // scratch in the staging area: words[2], done[2], flags, first[2]
  uint32_t* w = reinterpret_cast<uint32_t*>(ctx->stage);
  const uint32_t host[7] = {0u, 0u, 0u, 0u, 0u, 0u, 4u * kPersistThreads};
  CK(cudaMemcpyAsync(w, host, sizeof(host), cudaMemcpyHostToDevice, ctx->stream));
  PersistPlan S{};
  const int tasks = (4 + kPersistTilesPerTask - 1) / kPersistTilesPerTask;  // per pass
  S.pass[0] = PersistPass{kPDensity, kPersistThreads, 0, 4};
  S.pass[1] = PersistPass{kPDp, kPersistThreads, tasks, 4};
  S.npass = 2;
  S.tasks = 2 * tasks;
  S.nscenes = 1;
  S.stall_pass = 1;
  S.limit_ns = 2000000ull;  // 2 ms
  S.words = w;
  S.done = w + 2;
  S.flags = w + 4;
  S.first = w + 5;
  k_persist<true><<<8, kPersistThreads, 0, ctx->stream>>>(ctx->dev, ctx->fast, 4 * kPersistThreads, ctx->lstride, S,
                                                         PersistArrays{});
  if (int rc = check_launch(ctx, "selftest_persistent_wait_timeout")) return rc;
  CK(cudaMemcpyAsync(flags, S.flags, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PBF_OK;
}

int pbf_set_timing(pbf_ctx* ctx, int on) {
  if (!ctx) return PBF_ERR_ARG;
  ctx->timing = on != 0;
  return PBF_OK;
}

int pbf_reset_timing(pbf_ctx* ctx) {
  if (!ctx) return PBF_ERR_ARG;
  ctx->times.clear();
  ctx->time_order.clear();
  ctx->marks_used = 0;
  return PBF_OK;
}

int pbf_kernel_times(pbf_ctx* ctx, int max_kinds, const char** names, int64_t* launches, double* total_ms,
                     int* n_kinds) {
  if (!ctx) return PBF_ERR_ARG;
  if (int rc = harvest_times(ctx)) return rc;
  int i = 0;
  for (const auto& nm : ctx->time_order) {
    if (i >= max_kinds) break;
    const auto& t = ctx->times[nm];
    // names point at the static string literals the launches were tagged with
    for (const auto& m : ctx->marks)
      if (nm == m.name) {
        if (names) names[i] = m.name;
        break;
      }
    if (launches) launches[i] = t.first;
    if (total_ms) total_ms[i] = t.second;
    ++i;
  }
  if (n_kinds) *n_kinds = i;
  return PBF_OK;
}

// ---- launch shapes and the autotuner ----
int pbf_get_tuning(const pbf_ctx* ctx, pbf_tuning* out) {
  if (!ctx || !out) return PBF_ERR_ARG;
  *out = ctx->tune;
  return PBF_OK;
}

int pbf_set_tuning(pbf_ctx* ctx, const pbf_tuning* t) {
  if (!ctx || !t) return PBF_ERR_ARG;
  for (int f = 0; f < PBF_TUNE_FAMILIES; ++f)
    if (!shape_ok(t->lanes[f], t->block[f], t->staged[f]))
      return fail(ctx, PBF_ERR_ARG, "gather family %d: %d lanes x %d threads%s is not a supported shape "
                  "(lanes 2, 4 or 8, block 128 or 256; staged: 4 x 128)", f, t->lanes[f], t->block[f],
                  t->staged[f] ? " staged" : "");
  ctx->tune = *t;
  drop_graphs(ctx);
  return update_shapes(ctx);
}

namespace {
constexpr int kCandLanes[PBF_TUNE_CANDIDATES] = {4, 4, 8, 8, 2, 2, 4};
constexpr int kCandBlock[PBF_TUNE_CANDIDATES] = {128, 256, 128, 256, 128, 256, kStageThreads};
constexpr int kCandStaged[PBF_TUNE_CANDIDATES] = {0, 0, 0, 0, 0, 0, 1};

int family_of(const char* name) {
  if (!std::strcmp(name, "density_lambda") || !std::strcmp(name, "residual_check")) return PBF_TUNE_DENSITY;
  if (!std::strcmp(name, "dp_update")) return PBF_TUNE_DELTA_P;
  if (!std::strcmp(name, "viscosity") || !std::strcmp(name, "viscosity_final")) return PBF_TUNE_VISCOSITY;
  if (!std::strcmp(name, "vorticity")) return PBF_TUNE_VORTICITY;
  if (!std::strcmp(name, "apply_vorticity")) return PBF_TUNE_APPLY_VORTICITY;
  return -1;
}

// Device copies of the particle state an autotune must hand back unchanged.
struct StateSnapshot {
  std::vector<std::pair<void*, void*>> pairs;  // (live buffer, copy)
  std::vector<size_t> bytes;
  ~StateSnapshot() {
    for (auto& p : pairs) cudaFree(p.second);
  }
  int take(pbf_ctx* ctx, void* live, size_t nbytes) {
    void* copy = nullptr;
    if (cudaMalloc(&copy, nbytes) != cudaSuccess)
      return fail(ctx, PBF_ERR_CUDA, "autotune: cudaMalloc(%zu bytes) for the state copy failed", nbytes);
    pairs.emplace_back(live, copy);
    bytes.push_back(nbytes);
    CK(cudaMemcpyAsync(copy, live, nbytes, cudaMemcpyDeviceToDevice, ctx->stream));
    return PBF_OK;
  }
  int restore(pbf_ctx* ctx) {
    for (size_t i = 0; i < pairs.size(); ++i)
      CK(cudaMemcpyAsync(pairs[i].first, pairs[i].second, bytes[i], cudaMemcpyDeviceToDevice, ctx->stream));
    return PBF_OK;
  }
};
}  // namespace

int pbf_autotune(pbf_ctx* ctx, int steps, pbf_tuning* chosen, double* ms) {
  if (!ctx) return PBF_ERR_ARG;
  if (steps < 1) return fail(ctx, PBF_ERR_ARG, "autotune needs steps >= 1");
  if (ms) std::fill(ms, ms + PBF_TUNE_CANDIDATES * PBF_TUNE_FAMILIES, 0.0);
  if (ctx->params.solver == 1 && !ctx->mlp_ready)
    return fail(ctx, PBF_ERR_STATE, "learned solver without a network: call pbf_mlp_init or pbf_mlp_set");
  const size_t n = ctx->n;
  if (n == 0 || ctx->params.exact_math) {  // nothing to tune
    if (chosen) *chosen = ctx->tune;
    return PBF_OK;
  }
  StateSnapshot snap;
  int rc;
  if ((rc = snap.take(ctx, ctx->posH, n * sizeof(float4))) || (rc = snap.take(ctx, ctx->pstH, n * sizeof(float4))) ||
      (rc = snap.take(ctx, ctx->velH, n * sizeof(float4))) || (rc = snap.take(ctx, ctx->scrH, n * sizeof(float4))) ||
      (rc = snap.take(ctx, ctx->lamH, n * sizeof(float))) || (rc = snap.take(ctx, ctx->origH, n * sizeof(uint32_t))) ||
      (rc = snap.take(ctx, ctx->lamsumH, n * sizeof(float))) ||
      (rc = snap.take(ctx, ctx->fill_words, kFillWords * sizeof(uint32_t))))
    return rc;
  const bool timing = ctx->timing;
  const pbf_tuning before = ctx->tune;
  double t[PBF_TUNE_CANDIDATES][PBF_TUNE_FAMILIES] = {};
  double fill_ms[PBF_TUNE_CANDIDATES] = {};
  ctx->timing = true;
  auto finish = [&](int code) {
    ctx->timing = timing;
    ctx->times.clear();
    ctx->time_order.clear();
    ctx->marks_used = 0;
    ctx->lists_valid = false;
    drop_graphs(ctx);
    return code;
  };
  for (int c = 0; c < PBF_TUNE_CANDIDATES; ++c) {
    for (int f = 0; f < PBF_TUNE_FAMILIES; ++f) {
      ctx->tune.lanes[f] = kCandLanes[c];
      ctx->tune.block[f] = kCandBlock[c];
      ctx->tune.staged[f] = kCandStaged[c];
    }
    if ((rc = update_shapes(ctx)) || (rc = snap.restore(ctx))) return finish(rc);
    launch_step(ctx);  // untimed: first touch of this shape
    if ((rc = check_launch(ctx, "autotune")) || (rc = harvest_times(ctx))) return finish(rc);
    ctx->times.clear();
    ctx->time_order.clear();
    for (int i = 0; i < steps; ++i) launch_step(ctx);
    if ((rc = check_launch(ctx, "autotune")) || (rc = harvest_times(ctx))) return finish(rc);
    for (const auto& kv : ctx->times) {
      const int f = family_of(kv.first.c_str());
      if (f >= 0) t[c][f] += kv.second.second / steps;
      if (kv.first == "fill_neighbors") fill_ms[c] = kv.second.second / steps;
    }
  }
  // The fastest direct shape per family; then staging, for the families it
  // speeds up, only when those savings exceed what staging adds to the list
  // fill (the 16-bit lists and tile descriptors it then writes).
  pbf_tuning best = before;
  int pick[PBF_TUNE_FAMILIES];
  double direct_fill = 0.0;
  int ndirect = 0;
  for (int c = 0; c < PBF_TUNE_CANDIDATES; ++c)
    if (!kCandStaged[c]) {
      direct_fill += fill_ms[c];
      ++ndirect;
    }
  direct_fill /= ndirect > 0 ? ndirect : 1;
  double saved = 0.0;
  int staged_c = -1;
  for (int c = 0; c < PBF_TUNE_CANDIDATES; ++c)
    if (kCandStaged[c]) staged_c = c;
  for (int f = 0; f < PBF_TUNE_FAMILIES; ++f) {
    int bc = -1;
    for (int c = 0; c < PBF_TUNE_CANDIDATES; ++c)
      if (!kCandStaged[c] && (bc < 0 || t[c][f] < t[bc][f])) bc = c;
    pick[f] = bc;
    if (staged_c >= 0 && t[staged_c][f] > 0.0 && t[staged_c][f] < t[bc][f]) saved += t[bc][f] - t[staged_c][f];
  }
  const bool use_staged = staged_c >= 0 && saved > fill_ms[staged_c] - direct_fill;
  for (int f = 0; f < PBF_TUNE_FAMILIES; ++f) {
    int bc = pick[f];
    if (use_staged && t[staged_c][f] > 0.0 && t[staged_c][f] < t[bc][f]) bc = staged_c;
    if (t[bc][f] > 0.0) {  // a family the step never launches keeps its shape
      best.lanes[f] = kCandLanes[bc];
      best.block[f] = kCandBlock[bc];
      best.staged[f] = kCandStaged[bc];
    }
  }
  if (ms)
    for (int c = 0; c < PBF_TUNE_CANDIDATES; ++c)
      for (int f = 0; f < PBF_TUNE_FAMILIES; ++f) ms[c * PBF_TUNE_FAMILIES + f] = t[c][f];
  ctx->tune = best;
  if ((rc = update_shapes(ctx)) || (rc = snap.restore(ctx))) return finish(rc);
  CK(cudaStreamSynchronize(ctx->stream));
  if (chosen) *chosen = best;
  return finish(PBF_OK);
}

int pbf_launches_per_step(pbf_ctx* ctx, int64_t* out) {
  if (!ctx || !out) return PBF_ERR_ARG;
  *out = launches_per_step(ctx);
  return PBF_OK;
}

}  // extern "C"

// ============================================================================
// Neighbor search that allocates nothing
// ============================================================================
// For callers that may not allocate device memory themselves: hosts that own
// every device allocation through their own pool or a fixed budget, and
// callers that cannot afford the device-wide synchronisation cudaMalloc and
// cudaFree imply.  All working memory lives in the file-scope array below
// (PBF_NOALLOC_SCRATCH_BYTES, held on every GPU that loads the library until
// the process exits); the caller passes only its inputs and outputs.
// The steps are the regular neighbor search's:
//   hash      bin key and (index << 32 | index) at the caller's index, plus
//             the bin histogram (calculate_bins, neighbors.h:120-125)
//   bounds    exclusive scan of the histogram = begin/end of every bin
//             (find_bin_bounds, neighbors.h:137-148)
//   sort      the stable LSD radix passes of the regular path, ping-ponging
//             between two key/pair buffers of the array: O(n) per pass however
//             particles crowd into bins (sort_bins, neighbors.h:130-132)
//   gather    positions into sorted order, with their reference indices
//   runs      runs of bit-identical positions among consecutive sorted slots
//   fill      the lists in reference index space (fill_neighbors,
//             neighbors.h:197-230); a bin of more than kRunBin particles is
//             walked run by run, one distance test per run
//   flags     the error word (out-of-grid or non-finite positions) copied to
//             the caller's flag word.
namespace {

constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kNaN = PBF_NOALLOC_MAX_PARTICLES;
constexpr size_t kNaB = PBF_NOALLOC_MAX_BINS;
constexpr size_t kNaParts = (kNaB + 1 + kScanTile - 1) / kScanTile;
constexpr size_t kNaTiles = (kNaN + kRadixTile - 1) / kRadixTile;
constexpr size_t kNaHist = (size_t)kRadixDigits * kNaTiles;
constexpr size_t kNaHistParts = (kNaHist + 1 + kScanTile - 1) / kScanTile;
// layout of the scratch array (byte offsets)
constexpr size_t kOffCount = 0;
constexpr size_t kOffStart = align_up(kOffCount + 4 * kNaB);
constexpr size_t kOffParts = align_up(kOffStart + 4 * (kNaB + 1));
constexpr size_t kOffKeyA = align_up(kOffParts + 4 * kNaParts);
constexpr size_t kOffKeyB = align_up(kOffKeyA + 4 * kNaN);
constexpr size_t kOffPairA = align_up(kOffKeyB + 4 * kNaN);
constexpr size_t kOffPairB = align_up(kOffPairA + 8 * kNaN);
constexpr size_t kOffHist = align_up(kOffPairB + 8 * kNaN);
constexpr size_t kOffHistOff = align_up(kOffHist + 4 * kNaHist);
constexpr size_t kOffHistParts = align_up(kOffHistOff + 4 * (kNaHist + 1));
constexpr size_t kOffRunEnd = align_up(kOffHistParts + 4 * kNaHistParts);
constexpr size_t kOffSortedX = align_up(kOffRunEnd + 4 * kNaN);
constexpr size_t kOffSortedId = align_up(kOffSortedX + 16 * kNaN);
constexpr size_t kOffErr = align_up(kOffSortedId + 4 * kNaN);
constexpr size_t kNoallocBytes = align_up(kOffErr + 4);
static_assert(kNoallocBytes == PBF_NOALLOC_SCRATCH_BYTES, "PBF_NOALLOC_SCRATCH_BYTES in pbf.h is stale");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// Device address of g_noalloc_scratch per device, looked up once per device
// (host code must not use the symbol itself as an address).
std::mutex g_noalloc_mu;
void* g_noalloc_addr[128] = {nullptr};

// calculate_bins over caller AoS positions (neighbors.h:120-125), the sort's
// input at the caller's index and the bin histogram (one atomic per distinct
// bin of a warp).
__global__ void k_noalloc_hash(Dev P, int n, const float* __restrict__ x, uint32_t* key, unsigned long long* pair,
                               uint32_t* cell_count, uint32_t* err) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  uint32_t k;
  if (!pbf::bin_of(P, pbf::region_of(P, 0), x[3 * (size_t)a], x[3 * (size_t)a + 1], x[3 * (size_t)a + 2], k))
    atomicOr(err, PBF_FLAG_KEY_RANGE);
  key[a] = k;
  pair[a] = ((unsigned long long)a << 32) | (unsigned long long)a;
  const unsigned peers = __match_any_sync(__activemask(), k);
  if ((peers & ((1u << (threadIdx.x & 31)) - 1u)) == 0u) atomicAdd(&cell_count[k], (uint32_t)__popc(peers));
}

__global__ void k_noalloc_gather(int n, const unsigned long long* __restrict__ pairs, const float* __restrict__ x,
                                 float4* sorted_x, uint32_t* sorted_id) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const unsigned long long pr = pairs[b];
  const size_t a = (size_t)(pr & 0xffffffffull);
  sorted_x[b] = make_float4(x[3 * a], x[3 * a + 1], x[3 * a + 2], 0.0f);
  sorted_id[b] = (uint32_t)(pr >> 32);
}

// A crowded bin [q0, q1) run by run (runs of bit-identical positions from
// k_runs): one distance test per run; on a hit the run's particles are
// appended in order, the particle's own slot left out, while the list has
// room.  Equal positions give equal tests, so the list is the one-by-one
// walk's.  Returns the new length.
__device__ __noinline__ int noalloc_fill_runs(float px, float py, float pz, float s2, int cap, uint32_t self,
                                              uint32_t q0, uint32_t q1, const float4* __restrict__ pst,
                                              const uint32_t* __restrict__ run_end,
                                              const uint32_t* __restrict__ sorted_id, int32_t* row, int count) {
  for (uint32_t q = q0; q < q1;) {
    const float4 xq = pst[q];
    const uint32_t qe = min(run_end[q], q1);
    const float d2 = pbf::mag2<true>(pbf::xsub(px, xq.x), pbf::xsub(py, xq.y), pbf::xsub(pz, xq.z));
    if (d2 < s2) {
      for (uint32_t r = q; r < qe && count < cap; ++r) {
        if (r == self) continue;
        row[count++] = (int32_t)sorted_id[r];
      }
      if (count >= cap) break;
    }
    q = qe;
  }
  return count;
}

// The list fill writing straight into the caller's output in reference index
// space: out[id][k], -1 past the count.
__global__ void __launch_bounds__(kBlock) k_noalloc_fill(Dev P, int n, const float4* __restrict__ pst,
                                                         const uint32_t* __restrict__ sorted_id,
                                                         const uint32_t* __restrict__ cell_start,
                                                         const uint32_t* __restrict__ run_end, int32_t* out,
                                                         int32_t* out_cnt, uint32_t* err) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const float4 xp = pst[b];
  const int cap = P.cap;
  int32_t* row = out + (size_t)sorted_id[b] * cap;
  int count = 0;
  for (int i = -1; i < 2 && count < cap; i++) {
    const float cx = pbf::xadd(xp.x, pbf::xmul((float)i, P.s));
    for (int j = -1; j < 2 && count < cap; j++) {
      const float cy = pbf::xadd(xp.y, pbf::xmul((float)j, P.s));
      for (int k = -1; k < 2 && count < cap; k++) {
        const float cz = pbf::xadd(xp.z, pbf::xmul((float)k, P.s));
        uint32_t nb;
        if (!pbf::bin_of(P, pbf::region_of(P, 0), cx, cy, cz, nb)) {
          atomicOr(err, PBF_FLAG_KEY_RANGE);
          continue;
        }
        const uint32_t q0 = cell_start[nb], q1 = cell_start[nb + 1];
        if (q1 - q0 > kRunBin) {
          count = noalloc_fill_runs(xp.x, xp.y, xp.z, P.s2, cap, (uint32_t)b, q0, q1, pst, run_end, sorted_id,
                                    row, count);
          continue;
        }
        for (uint32_t q = q0; q < q1; ++q) {
          if (q == (uint32_t)b) continue;
          const float4 xq = pst[q];
          const float d2 = pbf::mag2<true>(pbf::xsub(xp.x, xq.x), pbf::xsub(xp.y, xq.y), pbf::xsub(xp.z, xq.z));
          if (d2 < P.s2) {
            row[count] = (int32_t)sorted_id[q];
            if (++count >= cap) break;
          }
        }
      }
    }
  }
  for (int k = count; k < cap; ++k) row[k] = -1;
  out_cnt[sorted_id[b]] = count;
}

}  // namespace

extern "C" int pbf_find_neighbors_noalloc(const pbf_params* p, const float* d_x, size_t n, int32_t* d_nbr,
                                          int32_t* d_cnt, uint32_t* d_flags, void* stream_handle) {
  if (!p || (n && (!d_x || !d_nbr || !d_cnt))) return fail(nullptr, PBF_ERR_ARG, "null argument");
  if (n > PBF_NOALLOC_MAX_PARTICLES)
    return fail(nullptr, PBF_ERR_CAPACITY, "pbf_find_neighbors_noalloc: %zu particles exceed the maximum of %d",
                n, PBF_NOALLOC_MAX_PARTICLES);
  Dev d;
  int64_t dims[3];
  if (int rc = make_dev(nullptr, *p, d, dims)) return rc;
  if (d.nbins > PBF_NOALLOC_MAX_BINS)
    return fail(nullptr, PBF_ERR_CAPACITY, "pbf_find_neighbors_noalloc: grid of %d bins exceeds the maximum of %d",
                d.nbins, PBF_NOALLOC_MAX_BINS);
  cudaStream_t s = static_cast<cudaStream_t>(stream_handle);
  cudaError_t e;
  if (n == 0) {
    if (d_flags && (e = cudaMemsetAsync(d_flags, 0, 4, s)) != cudaSuccess)
      return fail(nullptr, PBF_ERR_CUDA, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    return PBF_OK;
  }
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 128)
    return fail(nullptr, PBF_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  unsigned char* base;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr)
        return fail(nullptr, PBF_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
      g_noalloc_addr[dev] = ptr;
    }
    base = static_cast<unsigned char*>(g_noalloc_addr[dev]);
  }
  auto* cell_count = reinterpret_cast<uint32_t*>(base + kOffCount);
  auto* cell_start = reinterpret_cast<uint32_t*>(base + kOffStart);
  auto* parts = reinterpret_cast<uint32_t*>(base + kOffParts);
  uint32_t* kin = reinterpret_cast<uint32_t*>(base + kOffKeyA);
  uint32_t* kout = reinterpret_cast<uint32_t*>(base + kOffKeyB);
  auto* vin = reinterpret_cast<unsigned long long*>(base + kOffPairA);
  auto* vout = reinterpret_cast<unsigned long long*>(base + kOffPairB);
  auto* hist = reinterpret_cast<uint32_t*>(base + kOffHist);
  auto* hist_off = reinterpret_cast<uint32_t*>(base + kOffHistOff);
  auto* hist_parts = reinterpret_cast<uint32_t*>(base + kOffHistParts);
  auto* run_end = reinterpret_cast<uint32_t*>(base + kOffRunEnd);
  auto* sorted_x = reinterpret_cast<float4*>(base + kOffSortedX);
  auto* sorted_id = reinterpret_cast<uint32_t*>(base + kOffSortedId);
  auto* err = reinterpret_cast<uint32_t*>(base + kOffErr);
  // The array keeps the previous call's contents: clear what must start at
  // zero (the histogram and the error word; every other buffer is written in
  // full before it is read).
  e = cudaMemsetAsync(cell_count, 0, 4 * (size_t)d.nbins, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, 4, s);
  if (e != cudaSuccess) return fail(nullptr, PBF_ERR_CUDA, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
  const int nn = (int)n, g = blocks_for(n);
  const int nparts = (int)(((size_t)d.nbins + 1 + kScanTile - 1) / kScanTile);
  k_noalloc_hash<<<g, kBlock, 0, s>>>(d, nn, d_x, kin, vin, cell_count, err);
  k_scan_reduce<<<nparts, kScanThreads, 0, s>>>(cell_count, d.nbins, parts);
  k_scan_partials<<<1, kScanThreads, 0, s>>>(parts, nparts);
  k_scan_apply<<<nparts, kScanThreads, 0, s>>>(cell_count, d.nbins, parts, cell_start);
  const int tiles = (int)(((size_t)n + kRadixTile - 1) / kRadixTile);
  const int hm = kRadixDigits * tiles;
  const int hp = (int)(((size_t)hm + 1 + kScanTile - 1) / kScanTile);
  const int passes = radix_passes_for(d.nbins);
  for (int pass = 0; pass < passes; ++pass) {
    const int shift = pass * kRadixBits;
    const bool last = pass == passes - 1;
    k_radix_hist<<<tiles, kRadixThreads, 0, s>>>(kin, nn, shift, tiles, hist);
    k_scan_reduce<<<hp, kScanThreads, 0, s>>>(hist, hm, hist_parts);
    k_scan_partials<<<1, kScanThreads, 0, s>>>(hist_parts, hp);
    k_scan_apply<<<hp, kScanThreads, 0, s>>>(hist, hm, hist_parts, hist_off);
    k_radix_scatter<<<tiles, kRadixThreads, 0, s>>>(kin, vin, nn, shift, tiles, hist_off, last ? nullptr : kout,
                                                   vout);
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  k_noalloc_gather<<<g, kBlock, 0, s>>>(nn, vin, d_x, sorted_x, sorted_id);
  k_runs<<<blocks_for(n, kRunBlock), kRunBlock, 0, s>>>(nn, sorted_x, run_end, nullptr);
  k_noalloc_fill<<<g, kBlock, 0, s>>>(d, nn, sorted_x, sorted_id, cell_start, run_end, d_nbr, d_cnt, err);
  if (d_flags) e = cudaMemcpyAsync(d_flags, err, 4, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail(nullptr, PBF_ERR_CUDA, "noalloc neighbor search launch: %s", cudaGetErrorString(e));
  return PBF_OK;
}
