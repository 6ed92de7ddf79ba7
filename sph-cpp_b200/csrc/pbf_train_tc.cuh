// Training of the warm-start network on the 5th-generation tensor cores
// (sm_100a): the forward pass, the backward data GEMM and both weight-gradient
// GEMMs of one 128-sample tile as tcgen05.mma with BF16 operands in shared
// memory and FP32 accumulators in tensor memory.  The weight gradients stay
// in TMEM across all the tiles a CTA takes and go to global memory once, at
// the end of the launch.
//
// Per tile (s = sample of the tile's row, n/k = hidden units, f = features):
//   MMA1  Z1[s][n]  = X[s][f] . W1[n][f]          M128 N64 K16    (A sX,   B sW1)
//   epilogue 1: H1 = GELU(Z1 + b1)  -> sH1 [s][k] and sH1T [k][s]
//   MMA2  Z2[s][n]  = H1[s][k] . W2[n][k]         M128 N64 K64    (A sH1,  B sW2)
//   epilogue 2: y = GELU(Z2 + b2) . w3 + b3, dy = 2 (y - t) / B,
//               dZ2 = dy w3 GELU'(Z2 + b2)  -> sD2 [s][n] and sD2T [n][s];
//               dw3, db2, db3 and the loss summed per CTA
//   MMA3  dH1[s][k] = dZ2[s][n] . W2T[k][n]       M128 N64 K64    (A sD2,  B sW2T)
//   MMA4  dW2[n][k] += dZ2T[n][s] . H1T[k][s]     M128 N64 K128   (A sD2T, B sH1T; rows 64..127 of A zero)
//   epilogue 3: dZ1 = dH1 GELU'(Z1 + b1)  -> sD1T [n][s]; db1 summed
//   MMA5  dW1[n][f] += dZ1T[n][s] . XT[f][s]      M128 N16 K128   (A sD1T, B sXT;  rows 64..127 of A zero)
// TMEM columns: Z1 0..63, Z2 64..127, dH1 128..191, dW2 192..255, dW1 256..271
// (512 allocated; the kernel's shared memory keeps it to one CTA per SM).
// Operand layouts and descriptors are those of pbf_mlp_tc.cuh (K-major, no
// swizzle, core matrices 128 B apart along K, K/8 * 128 B along M/N).  Every
// wait on the MMAs' mbarrier is bounded; a wait that gives up raises
// PBF_FLAG_WAIT_TIMEOUT, leaves the tile loop on every thread, and the TMEM
// is freed.
#pragma once
#include "pbf_learn.cuh"
#include "pbf_mlp_tc.cuh"

namespace pbf {
namespace tt {

constexpr int kCols = 512;  // TMEM columns allocated
constexpr uint32_t kIdescM128N16 = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

// Shared-memory operand offsets (bytes, 1024-aligned) of the dynamic buffer.
constexpr uint32_t kX = 0;                                  // [128][16]
constexpr uint32_t kXT = kX + 128 * 16 * 2;                 // [16][128]
constexpr uint32_t kW1 = kXT + 16 * 128 * 2;                // [64][16]
constexpr uint32_t kW2 = kW1 + 64 * 16 * 2;                 // [64][64]
constexpr uint32_t kW2T = kW2 + 64 * 64 * 2;                // [64][64]
constexpr uint32_t kH1 = kW2T + 64 * 64 * 2;                // [128][64]
constexpr uint32_t kH1T = kH1 + 128 * 64 * 2;               // [64][128]
constexpr uint32_t kD2 = kH1T + 64 * 128 * 2;               // [128][64]
constexpr uint32_t kD2T = kD2 + 128 * 64 * 2;               // [128][128], rows 64..127 zero
constexpr uint32_t kD1T = kD2T + 128 * 128 * 2;             // [128][128], rows 64..127 zero
constexpr uint32_t kSmemBytes = kD1T + 128 * 128 * 2;       // 141,312
static_assert(kX % 1024 == 0 && kXT % 1024 == 0 && kW1 % 1024 == 0 && kW2 % 1024 == 0 && kW2T % 1024 == 0 &&
                  kH1 % 1024 == 0 && kH1T % 1024 == 0 && kD2 % 1024 == 0 && kD2T % 1024 == 0 && kD1T % 1024 == 0,
              "operand alignment");

__device__ __forceinline__ void tmem_alloc512(uint32_t slot) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(kCols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free512(uint32_t taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kCols) : "memory");
}

__device__ __forceinline__ void st_bf16(uint8_t* base, uint32_t off, float v) {
  *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

// Sum of v over the 32 lanes of the warp (every lane gets it).
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace tt

// Gradient of L = mean over the batch of (y - target)^2, added into grad
// (fp32, canonical order) and L into *loss.  NORMALIZE: raw features are
// normalised here (else already normalised); SAMPLE: rows drawn from the
// n_data recorded rows by the counter-based hash sample_row (else rows
// 0..batch-1); targets = labels * inv_label_scale.  A persistent grid, one
// 256-thread CTA per SM: two threads per sample row, each for half the
// columns.
template <bool NORMALIZE, bool SAMPLE, bool NO_ARRIVE = false>
__global__ void __launch_bounds__(tc::kThreads, 1) k_mlp_grad_tc(MlpDev M, const float* __restrict__ feats,
                                                                const float* __restrict__ labels, int n_data,
                                                                int batch, uint64_t seed, float inv_label_scale,
                                                                float* grad, float* loss, uint32_t* err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ float sb1[kMlpH], sb2[kMlpH], sw3[kMlpH];
  __shared__ float gb1[kMlpH], gb2[kMlpH], gw3[kMlpH], half2[2][tc::kRows];
  __shared__ float gloss, gb3;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ int fail;
  namespace T = tc;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row = tid & (T::kRows - 1), h = tid >> 7;
  const int tiles = (batch + T::kRows - 1) / T::kRows;
  // weights (BF16 operand copies), biases, zeroed sums and padding rows
  for (int i = tid; i < kMlpH * 2; i += T::kThreads) {
    const int r = i >> 1, kc = (i & 1) * 8;
    *reinterpret_cast<uint4*>(sm + tt::kW1 + T::core_off(r, kc, kMlpInPad)) =
        *reinterpret_cast<const uint4*>(M.w1 + r * kMlpInPad + kc);
  }
  for (int i = tid; i < kMlpH * 8; i += T::kThreads) {
    const int r = i >> 3, kc = (i & 7) * 8;
    *reinterpret_cast<uint4*>(sm + tt::kW2 + T::core_off(r, kc, kMlpH)) =
        *reinterpret_cast<const uint4*>(M.w2 + r * kMlpH + kc);
    *reinterpret_cast<uint4*>(sm + tt::kW2T + T::core_off(r, kc, kMlpH)) =
        *reinterpret_cast<const uint4*>(M.w2t + r * kMlpH + kc);
  }
  for (int i = tid; i < 64 * 128 / 8; i += T::kThreads) {  // rows 64..127 of the transposed A operands
    const int r = 64 + i / 16, kc = (i % 16) * 8;
    *reinterpret_cast<uint4*>(sm + tt::kD2T + T::core_off(r, kc, 128)) = make_uint4(0u, 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(sm + tt::kD1T + T::core_off(r, kc, 128)) = make_uint4(0u, 0u, 0u, 0u);
  }
  if (tid < kMlpH) {
    sb1[tid] = M.b1[tid];
    sb2[tid] = M.b2[tid];
    sw3[tid] = M.w3[tid];
    gb1[tid] = gb2[tid] = gw3[tid] = 0.0f;
  }
  const uint32_t bar = T::smem_u32(&mbar);
  if (tid == 0) {
    T::bar_init(bar, 1);
    fail = 0;
    gloss = gb3 = 0.0f;
  }
  if (warp == 0) tt::tmem_alloc512(T::smem_u32(&tslot));
  T::fence_before_sync();
  __syncthreads();
  T::fence_after_sync();
  const uint32_t tmem = tslot;
  const uint32_t lanes = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(32 * h);
  const uint32_t s0 = T::smem_u32(sm);
  const float b3 = M.b3[0];
  const float inv_b = 1.0f / (float)batch;
  uint32_t phase = 0;
  bool first = true;
  auto wait = [&]() {
    if (!T::bar_wait(bar, phase)) fail = 1;
    phase ^= 1u;
    __syncthreads();
  };
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int s = tile * T::kRows + row;
    const bool ok = s < batch;
    const int src = ok ? sample_row<SAMPLE>(seed, s, n_data) : 0;
    // features: half h holds columns 8h..8h+7 (12..15 are zero)
    float f[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = 8 * h + j;
      float x = 0.0f;
      if (ok && k < kMlpIn) {
        x = feats[(size_t)src * kMlpIn + k];
        if (NORMALIZE) x = (x - M.feat_mean[k]) * M.feat_inv_std[k];
      }
      f[j] = x;
    }
    *reinterpret_cast<uint4*>(sm + tt::kX + T::core_off(row, 8 * h, kMlpInPad)) =
        make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]),
                   pack_bf16x2(f[6], f[7]));
#pragma unroll
    for (int j = 0; j < 8; ++j) tt::st_bf16(sm, tt::kXT + T::core_off(8 * h + j, row, 128), f[j]);
    const float target = ok ? labels[src] * inv_label_scale : 0.0f;
    T::fence_proxy_async();
    T::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      T::fence_after_sync();
      if (!NO_ARRIVE) {
        T::mma_bf16(tmem, T::smem_desc(s0 + tt::kX, 128, 256), T::smem_desc(s0 + tt::kW1, 128, 256),
                    T::kIdescM128N64, 0u);
        T::mma_commit(bar);
      }
    }
    wait();
    if (fail) break;
    T::fence_after_sync();
    // epilogue 1: H1 = GELU(Z1 + b1)
#pragma unroll
    for (int c = 0; c < 32; c += 16) {
      float v[16];
      T::tmem_ld16(lanes + (uint32_t)c, v);
      const int c0 = 32 * h + c;
#pragma unroll
      for (int j = 0; j < 16; j += 8) {
        float g[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) g[q] = gelu(v[j + q] + sb1[c0 + j + q]);
        *reinterpret_cast<uint4*>(sm + tt::kH1 + T::core_off(row, c0 + j, kMlpH)) =
            make_uint4(pack_bf16x2(g[0], g[1]), pack_bf16x2(g[2], g[3]), pack_bf16x2(g[4], g[5]),
                       pack_bf16x2(g[6], g[7]));
#pragma unroll
        for (int q = 0; q < 8; ++q) tt::st_bf16(sm, tt::kH1T + T::core_off(c0 + j + q, row, 128), g[q]);
      }
    }
    T::fence_proxy_async();
    T::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      T::fence_after_sync();
      if (!NO_ARRIVE) {
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)
          T::mma_bf16(tmem + 64, T::smem_desc(s0 + tt::kH1 + 256u * ks, 128, 1024),
                      T::smem_desc(s0 + tt::kW2 + 256u * ks, 128, 1024), T::kIdescM128N64, ks > 0 ? 1u : 0u);
        T::mma_commit(bar);
      }
    }
    wait();
    if (fail) break;
    T::fence_after_sync();
    // epilogue 2: the output, its error, dZ2 and the layer-3 / bias-2 sums
    float z2[32];
    float part = 0.0f;
#pragma unroll
    for (int c = 0; c < 32; c += 16) {
      T::tmem_ld16(lanes + 64u + (uint32_t)c, z2 + c);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        z2[c + q] += sb2[32 * h + c + q];
        part = fmaf(gelu(z2[c + q]), sw3[32 * h + c + q], part);
      }
    }
    half2[h][row] = part;
    __syncthreads();
    const float y = half2[0][row] + half2[1][row] + b3;
    const float e = ok ? y - target : 0.0f;
    const float dy = 2.0f * e * inv_b;
    if (h == 0) {
      const float l = tt::warp_sum(e * e * inv_b), d3 = tt::warp_sum(dy);
      if (lane == 0) {
        atomicAdd(&gloss, l);
        atomicAdd(&gb3, d3);
      }
    }
#pragma unroll
    for (int c = 0; c < 32; c += 8) {
      float d[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int n = 32 * h + c + q;
        const float gw = tt::warp_sum(gelu(z2[c + q]) * dy);
        d[q] = dy * sw3[n] * gelu_grad(z2[c + q]);
        const float gb = tt::warp_sum(d[q]);
        if (lane == 0) {
          atomicAdd(&gw3[n], gw);
          atomicAdd(&gb2[n], gb);
        }
        tt::st_bf16(sm, tt::kD2T + T::core_off(n, row, 128), d[q]);
      }
      *reinterpret_cast<uint4*>(sm + tt::kD2 + T::core_off(row, 32 * h + c, kMlpH)) =
          make_uint4(pack_bf16x2(d[0], d[1]), pack_bf16x2(d[2], d[3]), pack_bf16x2(d[4], d[5]),
                     pack_bf16x2(d[6], d[7]));
    }
    T::fence_proxy_async();
    T::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      T::fence_after_sync();
      if (!NO_ARRIVE) {
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)  // dH1 = dZ2 W2
          T::mma_bf16(tmem + 128, T::smem_desc(s0 + tt::kD2 + 256u * ks, 128, 1024),
                      T::smem_desc(s0 + tt::kW2T + 256u * ks, 128, 1024), T::kIdescM128N64, ks > 0 ? 1u : 0u);
#pragma unroll
        for (int ks = 0; ks < 8; ++ks)  // dW2 += dZ2^T H1
          T::mma_bf16(tmem + 192, T::smem_desc(s0 + tt::kD2T + 256u * ks, 128, 2048),
                      T::smem_desc(s0 + tt::kH1T + 256u * ks, 128, 2048), T::kIdescM128N64,
                      (first && ks == 0) ? 0u : 1u);
        T::mma_commit(bar);
      }
    }
    wait();
    if (fail) break;
    T::fence_after_sync();
    // epilogue 3: dZ1 = dH1 GELU'(Z1 + b1) and the bias-1 sums
#pragma unroll
    for (int c = 0; c < 32; c += 16) {
      float dh[16], z1[16];
      T::tmem_ld16(lanes + 128u + (uint32_t)c, dh);
      T::tmem_ld16(lanes + (uint32_t)c, z1);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int n = 32 * h + c + q;
        const float d = dh[q] * gelu_grad(z1[q] + sb1[n]);
        const float gb = tt::warp_sum(d);
        if (lane == 0) atomicAdd(&gb1[n], gb);
        tt::st_bf16(sm, tt::kD1T + T::core_off(n, row, 128), d);
      }
    }
    T::fence_proxy_async();
    T::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      T::fence_after_sync();
      if (!NO_ARRIVE) {
#pragma unroll
        for (int ks = 0; ks < 8; ++ks)  // dW1 += dZ1^T X
          T::mma_bf16(tmem + 256, T::smem_desc(s0 + tt::kD1T + 256u * ks, 128, 2048),
                      T::smem_desc(s0 + tt::kXT + 256u * ks, 128, 2048), tt::kIdescM128N16,
                      (first && ks == 0) ? 0u : 1u);
        T::mma_commit(bar);
      }
    }
    wait();  // the next tile's features overwrite this MMA's B operand
    if (fail) break;
    T::fence_after_sync();
    first = false;
  }
  // the CTA's sums to global memory: weight gradients from TMEM (rows 0..63)
  if (!fail && !first) {
    if ((warp & 3) < 2) {  // TMEM lanes 0..63: the rows of dW2 and dW1
      const int n = row;
#pragma unroll
      for (int c = 0; c < 32; c += 16) {
        float v[16];
        T::tmem_ld16(lanes + 192u + (uint32_t)c, v);
#pragma unroll
        for (int q = 0; q < 16; ++q) atomicAdd(grad + kOffW2 + n * kMlpH + 32 * h + c + q, v[q]);
      }
      if (h == 0) {
        float v[16];
        T::tmem_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + 256u, v);
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) atomicAdd(grad + kOffW1 + n * kMlpIn + k, v[k]);
      }
    }
    if (tid < kMlpH) {
      atomicAdd(grad + kOffB1 + tid, gb1[tid]);
      atomicAdd(grad + kOffB2 + tid, gb2[tid]);
      atomicAdd(grad + kOffW3 + tid, gw3[tid]);
    }
    if (tid == 0) {
      atomicAdd(grad + kOffB3, gb3);
      atomicAdd(loss, gloss);
    }
  }
  if (fail && tid == 0) atomicOr(err, PBF_FLAG_WAIT_TIMEOUT);
  T::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    T::fence_after_sync();
    tt::tmem_free512(tmem);
  }
}

}  // namespace pbf
