// umma.cuh -- Blackwell (sm_100a) 5th-generation tensor-core primitives used
// by the learned coarse-grid correction: shared-memory matrix descriptors,
// the BF16 instruction descriptor, tcgen05.mma / commit, tensor-memory
// allocation and tcgen05.ld, written as inline PTX.
//
// Operand layouts are the "no swizzle" canonical layouts of the tcgen05
// matrix descriptors, in bytes (bf16 elements, a core matrix is 8 rows of
// 16 bytes):
//   K-major  (row r of M or N, k along K): (r%8)*16 + (r/8)*SBO + (k%8)*2 + (k/8)*LBO
//   MN-major (mn along M or N, k along K): (mn%8)*2 + (mn/8)*SBO + (k%8)*16 + (k/8)*LBO
// With SBO = 128 the rows of a K-major operand sit 16 bytes apart, so a
// shift by whole rows is a shift of the descriptor's start address.
#ifndef PMHD_LEARNED_UMMA_CUH
#define PMHD_LEARNED_UMMA_CUH

#include <cstdint>

#include "common.cuh"

namespace pmhd {
namespace umma {

// Shared-memory matrix descriptor: start address, leading-dimension byte
// offset (K-group stride), stride-dimension byte offset (8-row-group
// stride), all >> 4; bits 46-47 = 1 (descriptor version of sm_100);
// layout type 0 (no swizzle); base offset 0.
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 accumulator:
// D format bits 4-5 = 1 (f32), A format bits 7-9 = 1 (bf16), B format bits
// 10-12 = 1 (bf16), bit 15/16 = A/B MN-major, N>>3 at bits 17-22, M>>4 at
// bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D[tmem] (+)= A * B^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive on `bar` once every tcgen05.mma this thread issued has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Tensor-memory allocation (one full warp), result written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Eight consecutive 32-bit accumulator columns of this thread's lane (warp
// w of the CTA reads lanes 32w .. 32w+31), waiting for the load in the same
// statement so the values are never used early.
__device__ __forceinline__ void ld8(uint32_t taddr, float* v) {
  uint32_t r0, r1, r2, r3, r4, r5, r6, r7;
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7)
      : "r"(taddr)
      : "memory");
  v[0] = __uint_as_float(r0);
  v[1] = __uint_as_float(r1);
  v[2] = __uint_as_float(r2);
  v[3] = __uint_as_float(r3);
  v[4] = __uint_as_float(r4);
  v[5] = __uint_as_float(r5);
  v[6] = __uint_as_float(r6);
  v[7] = __uint_as_float(r7);
}

// Tensor-memory columns to allocate for `n` accumulator columns (a power of
// two >= 32).
__host__ __device__ constexpr uint32_t tmem_cols(int n) { return n <= 32 ? 32u : n <= 64 ? 64u : n <= 128 ? 128u : 256u; }

}  // namespace umma
}  // namespace pmhd

#endif  // PMHD_LEARNED_UMMA_CUH
