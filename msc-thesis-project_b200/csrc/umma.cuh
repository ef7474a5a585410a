// umma.cuh -- tcgen05 (5th-generation tensor core) helpers shared by the
// GEMM of mlp.cu and the fused proposal kernel of alp_learn.cu: shared
// memory and instruction descriptors for BF16 x BF16 -> FP32 MMAs with
// K-major operands in the no-swizzle canonical layout, and a bounded
// mbarrier wait.
#pragma once

#include <stdint.h>

namespace flsb200 {
constexpr uint32_t kSpinLimit = 1u << 26;  // bounded mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor, no swizzle, K-major (bit layout as CUTLASS
// cute::UMMA::SmemDescriptor: start >>4 [0,14), LBO >>4 [16,30), SBO >>4
// [32,46), version 1 [46,48), layout type 0 [61,64)).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor for kind::f16: F32 accumulator (bits 4-5 = 1),
// A and B BF16 (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// byte offset of element (r, k) of a tile of R rows (multiple of 8) in the
// canonical no-swizzle K-major layout: 8-row x 16-byte core matrices, row
// groups 128 B apart (SBO), 8-element K groups R/8 * 128 B apart (LBO)
__device__ __forceinline__ uint32_t canon_off(int r, int k, int R) {
  return (uint32_t)((((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// Waits (bounded) for phase `phase` of the mbarrier; true when it completed.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t phase) {
  uint32_t done = 0;
  for (uint32_t it = 0; it < kSpinLimit && !done; ++it) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(mbar)), "r"(phase));
  }
  return done != 0;
}

}  // namespace flsb200
