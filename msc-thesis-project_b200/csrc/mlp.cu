// mlp.cu -- BF16 tensor-core GEMM (tcgen05, accumulators in TMEM) used by
// the training and inference of the ALP parameter-proposal network
// (alp_learn.cu).  No counterpart in the reference.
//
// GEMM: C[M x N] = A[M x K] . B[N x K]^T, A and B bf16 row-major (K
// contiguous, "K-major"), FP32 accumulation.  One CTA of 128 threads owns a
// 128-row tile and the whole N (<= 256): per 64-wide K chunk the threads
// stage A and B into shared memory in the no-swizzle canonical K-major
// layout (8-row x 16-byte core matrices; SBO = 128 B between row groups,
// LBO = rows/8 * 128 B between 8-element K groups), one elected thread
// issues four tcgen05.mma (K = 16 each) and commits them to an mbarrier,
// and the accumulator stays in tensor memory until the epilogue reads it
// back with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = rows).
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "alp_learn.cuh"
#include "umma.cuh"

namespace flsb200 {

constexpr int kGemmThreads = 128;
constexpr int kKChunk = 64;

__global__ void __launch_bounds__(kGemmThreads) k_gemm_tn(const GemmArgs g) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * 128;
  const int NP = (g.N + 15) & ~15;          // padded N (multiple of 16)
  unsigned char *sA = smem;                  // 128 x 64 bf16 = 16 KB
  unsigned char *sB = smem + 128 * kKChunk * 2;  // NP x 64 bf16
  // TMEM columns: power of two >= 32 covering NP
  uint32_t ncols = 32;
  while ((int)ncols < NP) ncols <<= 1;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base_slot;
  const uint32_t idesc = umma_idesc_bf16(128, NP);
  uint32_t phase = 0;
  bool timed_out = false;

  for (int k0 = 0; k0 < g.K; k0 += kKChunk) {
    const int kc = min(kKChunk, g.K - k0);  // multiple of 16
    // stage A (128 x kc) and B (NP x kc), 8 bf16 (16 B) per store
    for (int i = tid; i < 128 * 8; i += kGemmThreads) {
      const int r = i >> 3, kg = i & 7;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (kg * 8 < kc && m0 + r < g.M)
        v = *reinterpret_cast<const uint4 *>(g.A + (size_t)(m0 + r) * g.lda + k0 + kg * 8);
      *reinterpret_cast<uint4 *>(sA + canon_off(r, kg * 8, 128)) = v;
    }
    for (int i = tid; i < NP * 8; i += kGemmThreads) {
      const int r = i >> 3, kg = i & 7;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (kg * 8 < kc && r < g.N)
        v = *reinterpret_cast<const uint4 *>(g.B + (size_t)r * g.ldb + k0 + kg * 8);
      *reinterpret_cast<uint4 *>(sB + canon_off(r, kg * 8, NP)) = v;
    }
    // generic-proxy smem writes -> visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
      const uint32_t lbo_a = (128 / 8) * 128, lbo_b = (uint32_t)(NP / 8) * 128;
      for (int s = 0; s < kc / 16; ++s) {
        const uint64_t da = umma_desc(a0 + s * 2 * lbo_a, lbo_a, 128);
        const uint64_t db = umma_desc(b0 + s * 2 * lbo_b, lbo_b, 128);
        const uint32_t acc = (k0 > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(&mbar)));
    }
    // every thread waits for the MMAs (bounded): they read the staged tiles
    uint32_t done = 0;
    for (uint32_t it = 0; it < kSpinLimit && !done; ++it) {
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}\n"
          : "=r"(done)
          : "r"(smem_u32(&mbar)), "r"(phase));
    }
    // the whole block agrees on giving up, so every thread takes the same
    // barriers below
    if (__syncthreads_or(!done)) {
      timed_out = true;
      break;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;");
  }

  if (!timed_out) {
    // epilogue: warp w reads rows 32w + lane, 16 columns per tcgen05.ld
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < NP; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
          "%14,%15}, [%16];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
            "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;");
      if (row < g.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = c0 + j;
          if (col >= g.N) break;
          float v = __uint_as_float(r[j]);
          if (g.bias) v += g.bias[col];
          if (g.relu) v = fmaxf(v, 0.0f);
          if (g.Cf) g.Cf[(size_t)row * g.ldc + col] = v;
          if (g.Cb) g.Cb[(size_t)row * g.ldc + col] = __float2bfloat16_rn(v);
        }
      }
    }
  } else {
    if (tid == 0 && g.status) atomicOr(g.status, 0x100u);
    // give the MMAs in flight a second bounded chance to finish before the
    // tensor memory they write is released
    uint32_t done = 0;
    for (uint32_t it = 0; it < kSpinLimit && !done; ++it) {
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}\n"
          : "=r"(done)
          : "r"(smem_u32(&mbar)), "r"(phase));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
  }
}

flsgpu_status gemm_tn(const GemmArgs &g, cudaStream_t s) {
  if (g.N <= 0 || g.N > 256 || (g.K % 16) != 0 || g.M <= 0)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "gemm shape M=%d N=%d K=%d", g.M, g.N, g.K);
  if (((uintptr_t)g.A % 16) || ((uintptr_t)g.B % 16) || (g.lda % 8) || (g.ldb % 8))
    return set_error(FLSGPU_ERR_MISALIGNED, "gemm operands must be 16-byte aligned");
  const int NP = (g.N + 15) & ~15;
  const size_t smem = (size_t)128 * kKChunk * 2 + (size_t)NP * kKChunk * 2;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_gemm_tn, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    attr = true;
  }
  k_gemm_tn<<<(g.M + 127) / 128, kGemmThreads, smem, s>>>(g);
  note_launch();
  return check_cuda(cudaGetLastError(), "k_gemm_tn launch");
}

}  // namespace flsb200

using namespace flsb200;

extern "C" {

// C (fp32, M x N, row stride ldc) = A (bf16, M x K) . B (bf16, N x K)^T
// [+ bias] [relu]; also writes bf16 to Cb when non-null.  Exposed for the
// numerics tests of the tensor-core path.
flsgpu_status flsgpu_gemm_bf16_tn(const void *A, int lda, const void *B, int ldb, int M, int N,
                                  int K, float *Cf, void *Cb, int ldc, const float *bias, int relu,
                                  uint32_t *d_status, flsgpu_stream stream) {
  GemmArgs g{reinterpret_cast<const __nv_bfloat16 *>(A), reinterpret_cast<const __nv_bfloat16 *>(B),
             lda, ldb, M, N, K, Cf, reinterpret_cast<__nv_bfloat16 *>(Cb), ldc, bias, relu,
             d_status};
  return gemm_tn(g, (cudaStream_t)stream);
}

}  // extern "C"
