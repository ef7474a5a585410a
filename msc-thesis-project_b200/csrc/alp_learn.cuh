// alp_learn.cuh -- shared definitions of the GPU ALP encoder and the learned
// (exponent, factor) proposal network.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "../../include/flsgpu_b200_ext.h"

namespace flsb200 {

// Classes: the 190 (exponent e, factor f) pairs with 0 <= f <= e <= 18
// (encoder.hpp:166-167 iterates them), numbered e*(e+1)/2 + f; class 190
// stands for ALP-RD; class 191 pads the output layer to 192.
constexpr int kClassRD = 190;
constexpr int kClasses = 191;
constexpr int kOut = 192;
constexpr int kFeatures = 64;
constexpr int kHidden = 128;

__host__ __device__ constexpr int pair_class(int e, int f) { return e * (e + 1) / 2 + f; }
__host__ __device__ inline int class_exp(int c) {
  int e = 0;
  while ((e + 1) * (e + 2) / 2 <= c) ++e;
  return e;
}
__host__ __device__ inline int class_fac(int c) {
  const int e = class_exp(c);
  return c - e * (e + 1) / 2;
}

// Per-vector encode parameters and sizes (the column's metadata arrays, plus
// the fill integer and the flags).
struct EncodeSlots {
  uint8_t *bw;
  uint64_t *base;
  int64_t *fill;      // integer stored at exception positions
  uint8_t *fac;
  uint8_t *exp;
  uint16_t *count;
  uint8_t *flags;     // 1 = the proposal fell back to the plain search; 2 = ALP-RD
  uint32_t *fb_list;  // vectors whose proposal fell back (mode 1)
  uint32_t *fb_count;
  size_t *blk_words;  // per 1024 vectors: offsets of the scan's blocks
  size_t *blk_exc;
  uint32_t *exc_mask; // per vector, 32 words: thread t's exception bits
};

// Launchers (alp_encode.cu)
flsgpu_status run_plain_labels(const double *vals, size_t n_vecs, int16_t *labels, int32_t *est,
                               cudaStream_t s);
// parameter choice (mode 0: plain search; 1: verified proposals with
// fallback) and analysis, scan of the per-vector sizes (totals[0] = packed
// words, totals[1] = exceptions), then packing into packed / exc / pos.
// With `rd` (hybrid columns) the vectors that call for ALP-RD are encoded
// into the ALP-RD workspace instead (rd->totals: right words, left words,
// exceptions; rd->scheme per vector).
struct RDWork;
flsgpu_status run_alp_encode(const double *vals, size_t n_vecs, int mode, const int16_t *cand,
                             int k_cand, int max_exc, const EncodeSlots &sl, size_t *off_words,
                             size_t *off_exc, size_t *totals, uint64_t *packed, double *exc,
                             uint16_t *pos, cudaStream_t s, RDWork *rd = nullptr);

// The f32 encoder (alp_encode_f32.cu): per-vector parameters and sizes.
struct Enc32Slots {
  uint8_t *bw, *fac, *exp;
  uint32_t *base;
  int32_t *fill;
  uint16_t *count;
  uint32_t *exc_mask;   // per vector, 32 words: thread t's exception bits
  uint32_t *sizes;      // [2][stride]: packed words, exceptions
  size_t stride;
  size_t *n_rd;         // vectors whose estimate reaches the ALP-RD limit
                        // (encoded as ALP all the same; counted)
};

flsgpu_status run_alp_encode_f32(const float *vals, size_t n_vecs, const Enc32Slots &sl,
                                 size_t *offs, size_t *blk, size_t bstride, size_t *totals,
                                 uint32_t *packed, float *exc, uint16_t *pos, cudaStream_t s);

struct GemmArgs {
  const __nv_bfloat16 *A;
  const __nv_bfloat16 *B;
  int lda, ldb;
  int M, N, K;          // N <= 256; K % 16 == 0
  float *Cf;            // optional fp32 output
  __nv_bfloat16 *Cb;    // optional bf16 output
  int ldc;
  const float *bias;    // optional, per column
  int relu;
  uint32_t *status;     // 0x100: an mbarrier wait gave up
};
flsgpu_status gemm_tn(const GemmArgs &g, cudaStream_t s);

}  // namespace flsb200
