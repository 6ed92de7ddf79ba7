// The warm-start network on the 5th-generation tensor cores (sm_100a):
// tcgen05.mma with BF16 operands in shared memory and FP32 accumulators in
// tensor memory (TMEM), one 128-row tile per MMA, the GELU epilogues read
// back with tcgen05.ld.
//
// Operand layout (both operands K-major, no swizzle): a "core matrix" is 8
// rows x 16 bytes (8 bf16 along K), stored contiguously (row stride 16 B);
// core matrices are 128 B apart along K (the leading byte offset, LBO) and
// K/8 * 128 B apart along M or N (the stride byte offset, SBO).  One
// kind::f16 MMA consumes K = 16 (two core matrices along K); a K = 64 operand
// is four MMAs whose descriptors start 256 B apart.
//
// Shared-memory descriptor (64 bit): start address >> 4 in bits [0,14),
// LBO >> 4 in [16,30), SBO >> 4 in [32,46), descriptor version 1 in [46,48),
// base offset 0, no swizzle (layout type 0 in [61,64)).
// Instruction descriptor (32 bit): accumulator F32 (1) in [4,6), A and B BF16
// (1) in [7,10) and [10,13), both K-major (bits 15, 16 clear), N >> 3 in
// [17,23), M >> 4 in [24,29).
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace pbf {
namespace tc {

constexpr int kRows = 128;        // M of one tile
constexpr int kThreads = 256;     // two threads per row, each for half the columns
constexpr int kTmemCols = 64;     // one accumulator, layer 2 reuses layer 1's columns
constexpr uint32_t kWaitPolls = 1u << 16;  // mbarrier polls before a wait gives up

// Byte offset of element (r, k) in a K-major bf16 operand with K columns.
__device__ __forceinline__ uint32_t core_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);
}

// M = 128, N = 64, BF16 x BF16 -> F32, both K-major.
constexpr uint32_t kIdescM128N64 = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n"
      :
      : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// Arrive on the mbarrier once every tcgen05 operation this thread issued is done.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void bar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the completion of the barrier phase with parity `phase`.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t phase) {
  for (uint32_t i = 0; i < kWaitPolls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Warp-wide (every lane of the warp): allocate / free kTmemCols columns.
__device__ __forceinline__ void tmem_alloc(uint32_t slot) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(kTmemCols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kTmemCols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes
// 32(w%4)..32(w%4)+31 of a 128-lane accumulator; taddr carries the warp's
// lane base).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace pbf
