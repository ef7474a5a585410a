// alp_learn.cu -- the learned (exponent, factor) proposal for the GPU ALP
// encoder: per-vector features, a 64 -> 128 -> 128 -> 192 MLP with BF16
// weights and FP32 accumulation on the tensor cores (mlp.cu), trained on the
// GPU with these kernels on labels from the plain sampling search
// (alp_encode.cu), and the encoder API that uses it.  No counterpart in the
// reference; it replaces encoder::init / find_top_k_combinations
// (src/alp/encoder.hpp:134-230, :400-406) as the source of candidate pairs,
// keeps the reference's second-level choice among candidates
// (encoder.hpp:237-300) and falls back to the plain search whenever the
// chosen pair leaves more than 3% exceptions, so decoding stays exact.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "alp_learn.cuh"
#include "rd_encode.cuh"
#include "umma.cuh"

namespace flsb200 {

static __constant__ double c_pow10_feat[17] = {1.0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7, 1e8,
                                               1e9,  1e10, 1e11, 1e12, 1e13, 1e14, 1e15, 1e16};

__device__ __forceinline__ float warp_sum_f(float x) {
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) x += __shfl_xor_sync(0xffffffffu, x, s);
  return x;
}
__device__ __forceinline__ float warp_min_f(float x) {
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) x = fminf(x, __shfl_xor_sync(0xffffffffu, x, s));
  return x;
}
__device__ __forceinline__ float warp_max_f(float x) {
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, s));
  return x;
}

// Bit planes: pl[k] = ballot(bit k of the lane's value).  plane_eq gives the
// lanes whose value equals `want`, plane_le those whose value is <= `want`;
// `want` differs per lane, so every lane counts its own histogram bin from
// the same few ballots instead of one ballot per bin.
template <int NB>
__device__ __forceinline__ uint32_t plane_eq(const uint32_t (&pl)[NB], uint32_t want) {
  uint32_t m = 0xffffffffu;
#pragma unroll
  for (int k = 0; k < NB; ++k) m &= ((want >> k) & 1u) ? pl[k] : ~pl[k];
  return m;
}
template <int NB>
__device__ __forceinline__ uint32_t plane_le(const uint32_t (&pl)[NB], uint32_t want) {
  uint32_t lt = 0, eq = 0xffffffffu;
#pragma unroll
  for (int k = NB - 1; k >= 0; --k) {
    const uint32_t b = (want >> k) & 1u;
    lt |= b ? (eq & ~pl[k]) : 0u;
    eq &= b ? pl[k] : ~pl[k];
  }
  return lt | eq;
}
// Order-preserving map of floats to unsigned keys (for integer warp min/max).
__device__ __forceinline__ uint32_t f_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float f_unkey(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
// A count below 2^23 as a float without a conversion instruction.
__device__ __forceinline__ float count_f(uint32_t c) {
  return __uint_as_float(0x4B000000u | c) - 8388608.0f;
}

// 64 features of a vector from its 32 samples (lane i holds value 32 i, the
// samples the search uses):
//   0..3   mean, deviation, min, max of log10|x| over the nonzero samples, / 10
//   4..6   fractions of zeros, negatives, non-finite samples
//   7..24  histogram of the decimal digits after the point (the smallest
//          d < 17 with x * 10^d integral, 17 when none)
//   25..41 histogram of trailing zero bits of the mantissa (/ 4; 16: none)
//   42..49 histogram of log10|x| in bins of 4 from -12
//   50..52 mean (/ 17 / 32 summed), max, min of the digits / 17
//   53     fraction with no digits after the point
//   54..57 mean, deviation of the binary exponent / 64; min, max / 1024
//   58..63 fractions with at most 2, 4, .., 12 digits after the point
// Lane t returns features t and t + 32 (lo[r], hi[r]) of R vectors at once
// (x[r] is the lane's sample of vector r), so the R computations interleave.
// Histogram bins come from bit-plane ballots and the integer statistics
// from warp integer reductions (each lane evaluates only its own two
// features); the floating-point sums keep a fixed shuffle order, so the
// training and the inference kernels see identical features.
template <int R>
__device__ __forceinline__ void vector_features(const double (&x)[R], int t, float (&lo)[R],
                                                float (&hi)[R]) {
  constexpr uint32_t kAll = 0xffffffffu;
  float l[R];
  int d[R], tz[R], e2[R];
  bool fin[R], nz[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const uint64_t bits = (uint64_t)__double_as_longlong(x[r]);
    fin[r] = isfinite(x[r]);
    const double a = fabs(x[r]);
    nz[r] = fin[r] && a > 0.0;
    // log10|x| from the binary exponent and the mantissa in [1, 2) (single
    // precision is far finer than the bf16 features; subnormals in double)
    const int ef = (int)((bits >> 52) & 0x7FF);
    const float mant = __uint_as_float(0x3F800000u | (uint32_t)((bits >> 29) & 0x7FFFFFu));
    l[r] = !nz[r] ? 0.0f
                  : ef ? __log10f(mant) + (float)(ef - 1023) * 0.30102999566f
                       : (float)log10(a);
    d[r] = 17;
    tz[r] = 53;
    if (nz[r]) {
      uint64_t mt = bits & 0xFFFFFFFFFFFFFull;
      if ((bits >> 52) & 0x7FF) mt |= 1ull << 52;
      tz[r] = __ffsll((long long)mt) - 1;
    }
    e2[r] = (int)((bits >> 52) & 0x7FF) - 1023;
  }
  // decimal digits after the point: the smallest dd < 17 with x * 10^dd
  // integral (17 when none, and for non-finite x); the scan stops once
  // every lane of the warp has its answer (most columns have few digits)
  {
    bool pend[R];
#pragma unroll
    for (int r = 0; r < R; ++r) pend[r] = fin[r];
#pragma unroll 1
    for (int dd = 0; dd < 17; ++dd) {
      const double p10 = c_pow10_feat[dd];
      bool any = false;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const double y = __dmul_rn(x[r], p10);
        if (pend[r] && fabs(y) < 9007199254740992.0 && y == rint(y)) {
          d[r] = dd;
          pend[r] = false;
        }
        any |= pend[r];
      }
      if (!__any_sync(kAll, any)) break;
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const uint32_t bnz = __ballot_sync(kAll, nz[r]);
    const uint32_t bzero = __ballot_sync(kAll, fin[r] && x[r] == 0.0);
    const uint32_t bneg = __ballot_sync(kAll, fin[r] && x[r] < 0.0);
    const uint32_t binf = __ballot_sync(kAll, !fin[r]);
    const uint32_t tzb = tz[r] >= 53 ? 16u : (uint32_t)min(15, tz[r] / 4);
    const uint32_t lb = (uint32_t)max(0, min(7, __float2int_rd((l[r] + 12.0f) * 0.25f)));
    uint32_t pd[5], pt[5], pm[3];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      pd[k] = __ballot_sync(kAll, ((uint32_t)d[r] >> k) & 1u);
      pt[k] = __ballot_sync(kAll, (tzb >> k) & 1u);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) pm[k] = __ballot_sync(kAll, (lb >> k) & 1u);
    // the lane's count features: lo slot t, hi slot 32 + t
    uint32_t mlo = t < 25 ? plane_eq(pd, (uint32_t)(t - 7)) : plane_eq(pt, (uint32_t)(t - 25));
    mlo = t == 4 ? bzero : t == 5 ? bneg : t == 6 ? binf : mlo;
    uint32_t mhi = t < 10 ? plane_eq(pt, (uint32_t)(t + 7)) : (plane_eq(pm, (uint32_t)(t - 10)) & bnz);
    mhi = t == 21 ? plane_eq(pd, 0u) : mhi;
    mhi = t >= 26 ? plane_le(pd, (uint32_t)(2 + 2 * (t - 26))) : mhi;

    // magnitude statistics over the nonzero samples
    const uint32_t nnzi = __popc(bnz);
    const float inv = nnzi > 0 ? 1.0f / count_f(nnzi) : 0.0f;
    const float mean_l = warp_sum_f(nz[r] ? l[r] : 0.0f) * inv;
    const float var_l = warp_sum_f(nz[r] ? (l[r] - mean_l) * (l[r] - mean_l) : 0.0f) * inv;
    const float lmin = f_unkey(__reduce_min_sync(kAll, nz[r] ? f_key(l[r]) : 0xffffffffu));
    const float lmax = f_unkey(__reduce_max_sync(kAll, nz[r] ? f_key(l[r]) : 0u));
    float num = t == 0 ? mean_l : t == 1 ? sqrtf(var_l) : t == 2 ? lmin : lmax;
    if (nnzi == 0 && t >= 2) num = 0.0f;
    lo[r] = t < 4 ? num / 10.0f : count_f(__popc(mlo)) * (1.0f / 32.0f);

    // digit and binary-exponent statistics (sums of small integers: exact)
    const int dsum = __reduce_add_sync(kAll, d[r]);
    const int dmax = __reduce_max_sync(kAll, d[r]);
    const int dmin = __reduce_min_sync(kAll, d[r]);
    const int esum = __reduce_add_sync(kAll, e2[r]);
    const int emin = __reduce_min_sync(kAll, e2[r]);
    const int emax = __reduce_max_sync(kAll, e2[r]);
    const float me = (float)esum / 32.0f;
    const float esd = sqrtf(warp_sum_f(((float)e2[r] - me) * ((float)e2[r] - me)) / 32.0f);
    const int ival = t == 18 ? dsum : t == 19 ? dmax : t == 20 ? dmin : t == 24 ? emin : emax;
    const float den = t == 18 ? 32.0f * 17.0f : t <= 20 ? 17.0f : 1024.0f;
    const float stat = t == 22 ? me / 64.0f : t == 23 ? esd / 64.0f : (float)ival / den;
    const bool hcount = t <= 17 || t == 21 || t >= 26;
    hi[r] = hcount ? count_f(__popc(mhi)) * (1.0f / 32.0f) : stat;
  }
}

__global__ void __launch_bounds__(256) k_features(const double *__restrict__ vals, size_t n_vecs,
                                                  __nv_bfloat16 *feat) {
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const double x[1] = {vals[v * VEC + 32 * t]};
    float lo[1], hi[1];
    vector_features<1>(x, t, lo, hi);
    feat[v * kFeatures + t] = __float2bfloat16_rn(lo[0]);
    feat[v * kFeatures + 32 + t] = __float2bfloat16_rn(hi[0]);
  }
}

using bf16 = __nv_bfloat16;

// ---- fused inference ------------------------------------------------------
// Features -> three layers -> top-k candidates of 128 vectors per tile in
// one persistent kernel (32 warps, one CTA per SM).  The bf16 weights are
// staged once per CTA in shared memory in the canonical K-major layout.  The
// CTA holds two teams of 16 warps, each with its own tile, activation tile,
// 256 tensor-memory columns, mbarrier and named barrier, so one team's
// feature arithmetic overlaps the other's MMAs and waits.  Per tile (row r =
// vector m0 + r): each warp of the team computes the features of 8 rows
// into the activation tile; one thread issues the MMAs of a layer (tcgen05,
// FP32 accumulators in tensor memory: layers 1 and 3 at columns 0.., layer
// 2 at 128..); warp w reads back tensor-memory lanes 32 (w % 4) .. +31
// (those rows) for column group (w % 16) / 4, adding bias + ReLU into the
// next activation tile, or, after layer 3, keeping the top-k of its group's
// logits, which the team's warps 0..3 merge per row.  The arithmetic is the
// layer-by-layer path's (the same MMAs in the same K order, bf16
// activations, fp32 logits, ties to the lower class), so the candidates are
// the same.
constexpr int kPropRows = 128;
constexpr int kPropThreads = 1024;
constexpr int kPropTeams = 2;                                 // tiles in flight per CTA
constexpr int kTeamThreads = kPropThreads / kPropTeams;       // 16 warps
constexpr int kPropGroups = kTeamThreads / kPropRows;         // column groups per row
constexpr int kTopMax = 4;
constexpr size_t kPropSmem =
    (size_t)(kHidden * kFeatures + kHidden * kHidden + kOut * kHidden +
             kPropTeams * kPropRows * kHidden) * 2 +
    (size_t)(kHidden + kHidden + kOut) * 4 +
    (size_t)kPropTeams * kPropGroups * kPropRows * kTopMax * (4 + 4);
static_assert(kPropSmem + 1024 <= 227 * 1024, "fused proposal: shared memory of one CTA");
static_assert(kPropTeams * 256 <= 512, "fused proposal: tensor-memory columns");

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;");
}

// Issues the K/16 MMAs of one layer: D[tmem] = A (128 x K, canonical, sA) .
// B (N x K, canonical, sB)^T, then commits them to the mbarrier.
__device__ __forceinline__ void issue_layer(uint32_t tmem_d, uint32_t sA, uint32_t sB, int N, int K,
                                            uint64_t *mbar) {
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t idesc = umma_idesc_bf16(kPropRows, N);
  const uint32_t lbo_a = (kPropRows / 8) * 128, lbo_b = (uint32_t)(N / 8) * 128;
  for (int s = 0; s < K / 16; ++s) {
    const uint64_t da = umma_desc(sA + s * 2 * lbo_a, lbo_a, 128);
    const uint64_t db = umma_desc(sB + s * 2 * lbo_b, lbo_b, 128);
    const uint32_t acc = s > 0 ? 1u : 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
  }
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
      smem_u32(mbar)));
}

// Columns [HC q, HC q + HC) (HC = 128 / column groups) of the row's hidden
// accumulator at tmem_col + bias, ReLU, to bf16 in the activation tile
// (K = 128 canonical layout), 8 columns per tensor-memory load.
__device__ __forceinline__ void hidden_epilogue(uint32_t tmem, int lanes, int q, int row,
                                                uint32_t tmem_col, const float *bias,
                                                unsigned char *sA) {
  constexpr int HC = kHidden / kPropGroups;
#pragma unroll
  for (int h = 0; h < HC / 8; ++h) {
    const int c0 = HC * q + 8 * h;
    uint32_t r[8];
    tmem_ld8(tmem + ((uint32_t)lanes << 16) + tmem_col + (uint32_t)c0, r);
    uint32_t packed[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float a = fmaxf(__uint_as_float(r[2 * j]) + bias[c0 + 2 * j], 0.0f);
      const float b = fmaxf(__uint_as_float(r[2 * j + 1]) + bias[c0 + 2 * j + 1], 0.0f);
      const __nv_bfloat162 hv = __floats2bfloat162_rn(a, b);
      packed[j] = *reinterpret_cast<const uint32_t *>(&hv);
    }
    *reinterpret_cast<uint4 *>(sA + canon_off(row, c0, kPropRows)) =
        make_uint4(packed[0], packed[1], packed[2], packed[3]);
  }
}

// Insertion into a list sorted by descending value; a value equal to one
// already listed goes behind it (candidates arrive in ascending class).
__device__ __forceinline__ void top_insert(float (&bv)[kTopMax], int (&bc)[kTopMax], int k, float val,
                                           int cls) {
#pragma unroll
  for (int q = 0; q < kTopMax; ++q) {
    if (q < k && cls >= 0 && (bc[q] < 0 || val > bv[q])) {
      const float tv = bv[q];
      const int tc = bc[q];
      bv[q] = val;
      bc[q] = cls;
      val = tv;
      cls = tc;
    }
  }
}

// Barrier of one team (named barrier 1 + team over its threads); team_any
// also returns whether any of them passed true.
__device__ __forceinline__ void team_sync(int team) {
  asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(kTeamThreads) : "memory");
}
__device__ __forceinline__ bool team_any(int team, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(team + 1), "r"(kTeamThreads)
      : "memory");
  return r != 0;
}

__global__ void __launch_bounds__(kPropThreads, 1)
    k_propose(const double *__restrict__ vals, size_t n_vecs, const bf16 *__restrict__ w1,
              const bf16 *__restrict__ w2, const bf16 *__restrict__ w3,
              const float *__restrict__ b1, const float *__restrict__ b2,
              const float *__restrict__ b3, int k, int16_t *cand, uint32_t *status) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar[kPropTeams];
  __shared__ uint32_t tmem_slot;
  unsigned char *sW1 = smem;
  unsigned char *sW2 = sW1 + kHidden * kFeatures * 2;
  unsigned char *sW3 = sW2 + kHidden * kHidden * 2;
  unsigned char *sA0 = sW3 + kOut * kHidden * 2;  // [teams][128 x 128 bf16]
  float *sb1 = reinterpret_cast<float *>(sA0 + kPropTeams * kPropRows * kHidden * 2);
  float *sb2 = sb1 + kHidden;
  float *sb3 = sb2 + kHidden;
  float *s_topv0 = sb3 + kOut;  // [teams][column groups][128][kTopMax]
  int *s_topc0 = reinterpret_cast<int *>(s_topv0 + kPropTeams * kPropGroups * kPropRows * kTopMax);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int kTeamWarps = kTeamThreads / 32;
  const int team = warp / kTeamWarps, tw = warp % kTeamWarps;
  // tensor-memory lanes 32 (warp % 4) .. +31 are the ones this warp may read
  const int lanes = 32 * (tw & 3), quarter = tw >> 2, row = lanes + lane;  // quarter: column group
  constexpr uint32_t kCols = 256 * kPropTeams;

  // weights and biases, once per CTA
  for (int i = tid; i < kHidden * kFeatures / 8; i += kPropThreads) {
    const int r = i / (kFeatures / 8), kg = i % (kFeatures / 8);
    *reinterpret_cast<uint4 *>(sW1 + canon_off(r, kg * 8, kHidden)) =
        *reinterpret_cast<const uint4 *>(w1 + (size_t)r * kFeatures + kg * 8);
  }
  for (int i = tid; i < kHidden * kHidden / 8; i += kPropThreads) {
    const int r = i / (kHidden / 8), kg = i % (kHidden / 8);
    *reinterpret_cast<uint4 *>(sW2 + canon_off(r, kg * 8, kHidden)) =
        *reinterpret_cast<const uint4 *>(w2 + (size_t)r * kHidden + kg * 8);
  }
  for (int i = tid; i < kOut * kHidden / 8; i += kPropThreads) {
    const int r = i / (kHidden / 8), kg = i % (kHidden / 8);
    *reinterpret_cast<uint4 *>(sW3 + canon_off(r, kg * 8, kOut)) =
        *reinterpret_cast<const uint4 *>(w3 + (size_t)r * kHidden + kg * 8);
  }
  for (int i = tid; i < kHidden; i += kPropThreads) {
    sb1[i] = b1[i];
    sb2[i] = b2[i];
  }
  for (int i = tid; i < kOut; i += kPropThreads) sb3[i] = b3[i];
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid < kPropTeams)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar[tid])), "r"(1));
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  // this team's accumulators (256 columns), activation tile, top-k scratch
  const uint32_t tmem = tmem_slot + 256u * (uint32_t)team;
  unsigned char *sA = sA0 + team * (kPropRows * kHidden * 2);
  float *s_topv = s_topv0 + team * (kPropGroups * kPropRows * kTopMax);
  int *s_topc = s_topc0 + team * (kPropGroups * kPropRows * kTopMax);
  uint64_t *mb = &mbar[team];
  const bool issuer = tw == 0 && lane == 0;
  const uint32_t aA = smem_u32(sA), aW1 = smem_u32(sW1), aW2 = smem_u32(sW2), aW3 = smem_u32(sW3);
  uint32_t phase = 0;
  bool failed = false;
  const size_t n_tiles = (n_vecs + kPropRows - 1) / kPropRows;
  constexpr int kRowsPerWarp = kPropRows / kTeamWarps;

  for (size_t tile = (size_t)blockIdx.x * kPropTeams + team; tile < n_tiles && !failed;
       tile += (size_t)gridDim.x * kPropTeams) {
    const size_t m0 = tile * kPropRows;
    // features of this warp's rows: lane j loads sample j of all of them
    // first (one round trip), then the warp works through them in pairs
    double xs[kRowsPerWarp];
#pragma unroll
    for (int i = 0; i < kRowsPerWarp; ++i) {
      const size_t v = m0 + tw * kRowsPerWarp + i;
      xs[i] = v < n_vecs ? vals[v * VEC + 32 * lane] : 0.0;
    }
#pragma unroll
    for (int i = 0; i < kRowsPerWarp; i += 2) {
      const double x2[2] = {xs[i], xs[i + 1]};
      float lo[2], hi[2];
      vector_features<2>(x2, lane, lo, hi);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int r = tw * kRowsPerWarp + i + q;
        *reinterpret_cast<bf16 *>(sA + canon_off(r, lane, kPropRows)) = __float2bfloat16_rn(lo[q]);
        *reinterpret_cast<bf16 *>(sA + canon_off(r, lane + 32, kPropRows)) =
            __float2bfloat16_rn(hi[q]);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;");
    asm volatile("tcgen05.fence::before_thread_sync;");
    team_sync(team);
    // layer 1 -> columns 0..127
    if (issuer) issue_layer(tmem, aA, aW1, kHidden, kFeatures, mb);
    if (team_any(team, !mbar_wait(mb, phase))) {
      failed = true;
      break;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;");
    hidden_epilogue(tmem, lanes, quarter, row, 0, sb1, sA);
    asm volatile("fence.proxy.async.shared::cta;");
    asm volatile("tcgen05.fence::before_thread_sync;");
    team_sync(team);
    // layer 2 -> columns 128..255
    if (issuer) issue_layer(tmem + 128, aA, aW2, kHidden, kHidden, mb);
    if (team_any(team, !mbar_wait(mb, phase))) {
      failed = true;
      break;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;");
    hidden_epilogue(tmem, lanes, quarter, row, 128, sb2, sA);
    asm volatile("fence.proxy.async.shared::cta;");
    asm volatile("tcgen05.fence::before_thread_sync;");
    team_sync(team);
    // layer 3 -> columns 0..191
    if (issuer) issue_layer(tmem, aA, aW3, kOut, kHidden, mb);
    if (team_any(team, !mbar_wait(mb, phase))) {
      failed = true;
      break;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;");
    // top-k of this group's share of the row's logits (LC classes from
    // LC q; class 191 is padding)
    {
      constexpr int LC = kOut / kPropGroups;
      float bv[kTopMax];
      int bc[kTopMax];
#pragma unroll
      for (int q = 0; q < kTopMax; ++q) {
        bv[q] = -INFINITY;
        bc[q] = -1;
      }
#pragma unroll
      for (int h = 0; h < LC / 8; ++h) {
        const int c0 = LC * quarter + 8 * h;
        uint32_t r[8];
        tmem_ld8(tmem + ((uint32_t)lanes << 16) + (uint32_t)c0, r);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int c = c0 + j;
          if (c < kClasses) top_insert(bv, bc, k, __uint_as_float(r[j]) + sb3[c], c);
        }
      }
#pragma unroll
      for (int q = 0; q < kTopMax; ++q) {
        s_topv[(quarter * kPropRows + row) * kTopMax + q] = bv[q];
        s_topc[(quarter * kPropRows + row) * kTopMax + q] = bc[q];
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    team_sync(team);
    if (quarter == 0) {
      // merge the groups in class order: a logit equal to one already
      // listed stays behind it
      float bv[kTopMax];
      int bc[kTopMax];
#pragma unroll
      for (int q = 0; q < kTopMax; ++q) {
        bv[q] = s_topv[row * kTopMax + q];
        bc[q] = s_topc[row * kTopMax + q];
      }
#pragma unroll
      for (int qq = 1; qq < kPropGroups; ++qq)
#pragma unroll
        for (int q = 0; q < kTopMax; ++q)
          top_insert(bv, bc, k, s_topv[(qq * kPropRows + row) * kTopMax + q],
                     s_topc[(qq * kPropRows + row) * kTopMax + q]);
      const size_t v = m0 + row;
      if (v < n_vecs)
        for (int q = 0; q < k; ++q) cand[v * k + q] = (int16_t)bc[q];
    }
    // the activation tile, the top-k scratch and tensor memory are reused
    team_sync(team);
  }
  if (failed) {
    if (issuer && status) atomicOr(status, 0x100u);
    mbar_wait(mb, phase);  // the MMAs in flight, bounded, before dealloc
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_slot), "r"(kCols));
}

// Softmax cross entropy over the 191 real classes of each row (class 191
// is padding): loss[row] and dZ = (softmax - onehot) / rows (bf16).
__global__ void k_softmax_ce(const float *__restrict__ z, const int16_t *__restrict__ labels,
                             int rows, float *loss, __nv_bfloat16 *dz) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int t = threadIdx.x & 31;
  if (row >= rows) return;
  const float *zr = z + (size_t)row * kOut;
  float m = -1e30f;
  for (int c = t; c < kClasses; c += 32) m = fmaxf(m, zr[c]);
  m = warp_max_f(m);
  float s = 0.0f;
  for (int c = t; c < kClasses; c += 32) s += __expf(zr[c] - m);
  s = warp_sum_f(s);
  const int y = labels[row];
  const float inv_rows = 1.0f / (float)rows;
  for (int c = t; c < kOut; c += 32) {
    float g = 0.0f;
    if (c < kClasses) g = (__expf(zr[c] - m) / s - (c == y ? 1.0f : 0.0f)) * inv_rows;
    dz[(size_t)row * kOut + c] = __float2bfloat16_rn(g);
  }
  if (t == 0) loss[row] = -(zr[y] - m - __logf(s));
}

// out[c][r] = in[r][c] (bf16), rows x cols -> cols x ld_out
__global__ void k_transpose_bf16(const __nv_bfloat16 *__restrict__ in, int rows, int cols,
                                 int ld_in, __nv_bfloat16 *out, int ld_out) {
  __shared__ __nv_bfloat16 tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    tile[i][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * ld_in + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (c < cols && r < rows) out[(size_t)c * ld_out + r] = tile[threadIdx.x][i];
  }
}

// dX (bf16) = dXf * (H > 0): the ReLU derivative applied to an fp32 gradient
__global__ void k_relu_back(const float *__restrict__ dxf, const __nv_bfloat16 *__restrict__ h,
                            int rows, int cols, __nv_bfloat16 *dx) {
  const size_t n = (size_t)rows * cols;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float g = __bfloat162float(h[i]) > 0.0f ? dxf[i] : 0.0f;
    dx[i] = __float2bfloat16_rn(g);
  }
}

// db[c] = sum over rows of g[r][c] (g bf16), one thread per column
// Column sums (bias gradients): a block of 32 x 32 threads per 32 columns;
// thread (c, y) adds rows y, y + 32, ... of column c, then the 32 partial
// sums of a column are added in shared memory.
__global__ void __launch_bounds__(1024) k_colsum_bf16(const __nv_bfloat16 *__restrict__ g,
                                                      int rows, int cols, float *db) {
  __shared__ float part[32][33];
  const int c = blockIdx.x * 32 + threadIdx.x, y = threadIdx.y;
  float s = 0.0f;
  if (c < cols)
    for (int r = y; r < rows; r += 32) s += __bfloat162float(g[(size_t)r * cols + c]);
  part[y][threadIdx.x] = s;
  __syncthreads();
  if (y == 0 && c < cols) {
    float t = 0.0f;
    for (int i = 0; i < 32; ++i) t += part[i][threadIdx.x];
    db[c] = t;
  }
}

// Adam on fp32 master parameters; refreshes the bf16 copy (and its
// transpose when wt != nullptr; rows x cols row-major).
__global__ void k_adam(float *w, const float *g, float *m, float *v, int n, float lr, float b1,
                       float b2, float eps, float c1, float c2, __nv_bfloat16 *wb,
                       __nv_bfloat16 *wt, int rows, int cols) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
  if (wt) {
    const int r = i / cols, c = i % cols;
    wt[(size_t)c * rows + r] = __float2bfloat16_rn(wi);
  }
}

__global__ void k_to_bf16(const float *w, int n, __nv_bfloat16 *wb, __nv_bfloat16 *wt, int rows,
                          int cols) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  wb[i] = __float2bfloat16_rn(w[i]);
  if (wt) {
    const int r = i / cols, c = i % cols;
    wt[(size_t)c * rows + r] = __float2bfloat16_rn(w[i]);
  }
}

// Top-k (k <= 4) classes of each row of the logits, best first; ties keep
// the smaller class.  One warp per row.
__global__ void k_topk(const float *__restrict__ z, int rows, int k, int16_t *cand) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int t = threadIdx.x & 31;
  if (row >= rows) return;
  const float *zr = z + (size_t)row * kOut;
  unsigned long long taken = 0ull, taken2 = 0ull, taken3 = 0ull, taken4 = 0ull;
  for (int j = 0; j < k; ++j) {
    float bv = -1e30f;
    int bc = 1 << 20;
    for (int c = t; c < kClasses; c += 32) {
      const int word = c >> 6, bit = c & 63;
      const unsigned long long tk = word == 0 ? taken : word == 1 ? taken2 : word == 2 ? taken3 : taken4;
      if ((tk >> bit) & 1ull) continue;
      const float val = zr[c];
      if (val > bv || (val == bv && c < bc)) {
        bv = val;
        bc = c;
      }
    }
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, bv, s);
      const int oc = __shfl_xor_sync(0xffffffffu, bc, s);
      if (ov > bv || (ov == bv && oc < bc)) {
        bv = ov;
        bc = oc;
      }
    }
    if (t == 0) cand[(size_t)row * k + j] = (int16_t)bc;
    const int word = bc >> 6, bit = bc & 63;
    if (word == 0) taken |= 1ull << bit;
    else if (word == 1) taken2 |= 1ull << bit;
    else if (word == 2) taken3 |= 1ull << bit;
    else taken4 |= 1ull << bit;
  }
}

}  // namespace flsb200

// ---------------------------------------------------------------------------
// host side: the encoder object
// ---------------------------------------------------------------------------
namespace {

using namespace flsb200;
using bf16 = __nv_bfloat16;

// parameter layout in one fp32 array (also the save-file payload)
constexpr int kW1 = kHidden * kFeatures, kB1 = kHidden;
constexpr int kW2 = kHidden * kHidden, kB2 = kHidden;
constexpr int kW3 = kOut * kHidden, kB3 = kOut;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kW1, kOffW2 = kOffB1 + kB1, kOffB2 = kOffW2 + kW2,
              kOffB2End = kOffB2 + kB2, kOffW3 = kOffB2End, kOffB3 = kOffW3 + kW3,
              kParams = kOffB3 + kB3;

template <typename T> T *dalloc(size_t n, flsgpu_status &st) {
  void *p = nullptr;
  if (st == FLSGPU_OK) st = check_cuda(cudaMalloc(&p, (n ? n : 1) * sizeof(T) + 16), "cudaMalloc");
  return static_cast<T *>(p);
}

}  // namespace

namespace flsb200 {
// A keyed permutation of [0, n): four Feistel rounds over 2 * half_bits
// bits (a bijection of [0, 4^half_bits)), applied again while the result is
// n or more (cycle walking; the domain is less than 4n, so few repeats, and
// the walk ends within the cycle of x).
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ uint32_t permute_index(uint32_t i, uint32_t n, int half_bits,
                                                  uint32_t key) {
  const uint32_t mask = (1u << half_bits) - 1u;
  const uint64_t domain = 1ull << (2 * half_bits);
  uint32_t x = i;
  for (uint64_t guard = 0; guard < domain; ++guard) {
    uint32_t l = x >> half_bits, r = x & mask;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t f = mix32(r ^ (key + 0x632BE5ABu * (uint32_t)k)) & mask;
      const uint32_t nl = r;
      r = l ^ f;
      l = nl;
    }
    x = (l << half_bits) | r;
    if (x < n) break;
  }
  return x;
}

// Row r of the epoch's training order is feature row permute_index(r):
// 64 bf16 features (eight 16-byte chunks, one per thread) and the label.
__global__ void __launch_bounds__(256) k_gather_rows(const __nv_bfloat16 *__restrict__ feat,
                                                     const int16_t *__restrict__ labels,
                                                     uint32_t n, size_t rows, int half_bits,
                                                     uint32_t key, __nv_bfloat16 *out_feat,
                                                     int16_t *out_lab) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * 8) return;
  const size_t r = i >> 3;
  const int chunk = (int)(i & 7);
  const uint32_t src = permute_index((uint32_t)r, n, half_bits, key);
  reinterpret_cast<uint4 *>(out_feat)[r * 8 + chunk] =
      reinterpret_cast<const uint4 *>(feat)[(size_t)src * 8 + chunk];
  if (chunk == 0) out_lab[r] = labels[src];
}
}  // namespace flsb200

struct flsgpu_alp_encoder {
  // parameters (fp32 master), Adam moments, gradients
  float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
  bf16 *w1b = nullptr, *w2b = nullptr, *w3b = nullptr;  // bf16 copies
  bf16 *w2t = nullptr, *w3t = nullptr;                  // bf16 transposes
  // activations of one batch
  int cap_rows = 0;
  bf16 *x = nullptr, *h1 = nullptr, *h2 = nullptr, *dz = nullptr;
  float *z = nullptr, *tmpf = nullptr, *loss = nullptr;
  bf16 *dh = nullptr, *t_a = nullptr, *t_b = nullptr;
  uint32_t *status = nullptr;
  int adam_t = 0;
  // encode workspaces (sized for cap_vecs vectors)
  size_t cap_vecs = 0;
  bf16 *feat = nullptr;
  int16_t *labels = nullptr, *cand = nullptr;
  EncodeSlots sl{};
  size_t *off_words = nullptr, *off_exc = nullptr, *totals = nullptr;
  uint64_t *packed = nullptr;
  double *exc = nullptr;
  uint16_t *pos = nullptr;
  size_t *exc_offs = nullptr, *vec_offs = nullptr;
  // ALP-RD encoder workspace (its column, and the RD part of hybrid columns)
  RDWork rd;
  // f32 encoder: per-vector sizes and offsets ([2][cap_vecs]), scan blocks
  uint32_t *f32_sizes = nullptr;
  size_t *f32_offs = nullptr, *f32_blk = nullptr, *f32_tot = nullptr;
};

namespace {

void free_acts(flsgpu_alp_encoder *e) {
  for (void *p : {(void *)e->x, (void *)e->h1, (void *)e->h2, (void *)e->dz, (void *)e->z,
                  (void *)e->tmpf, (void *)e->loss, (void *)e->dh, (void *)e->t_a, (void *)e->t_b})
    if (p) cudaFree(p);
  e->x = e->h1 = e->h2 = e->dz = e->dh = e->t_a = e->t_b = nullptr;
  e->z = e->tmpf = e->loss = nullptr;
  e->cap_rows = 0;
}

flsgpu_status ensure_rows(flsgpu_alp_encoder *e, int rows) {
  if (rows <= e->cap_rows) return FLSGPU_OK;
  free_acts(e);
  flsgpu_status st = FLSGPU_OK;
  const size_t r = (size_t)((rows + 127) / 128 * 128);
  e->x = dalloc<bf16>(r * kFeatures, st);
  e->h1 = dalloc<bf16>(r * kHidden, st);
  e->h2 = dalloc<bf16>(r * kHidden, st);
  e->dz = dalloc<bf16>(r * kOut, st);
  e->z = dalloc<float>(r * kOut, st);
  e->tmpf = dalloc<float>(r * kOut, st);
  e->loss = dalloc<float>(r, st);
  e->dh = dalloc<bf16>(r * kOut, st);
  e->t_a = dalloc<bf16>(r * kOut, st);
  e->t_b = dalloc<bf16>(r * kOut, st);
  if (st == FLSGPU_OK) e->cap_rows = (int)r;
  return st;
}

void free_enc(flsgpu_alp_encoder *e) {
  for (void *p : {(void *)e->feat, (void *)e->labels, (void *)e->cand, (void *)e->sl.fill,
                  (void *)e->sl.fb_list, (void *)e->sl.fb_count, (void *)e->sl.blk_words,
                  (void *)e->sl.blk_exc, (void *)e->sl.exc_mask,
                  (void *)e->sl.bw, (void *)e->sl.base,
                  (void *)e->sl.fac, (void *)e->sl.exp, (void *)e->sl.count, (void *)e->sl.flags,
                  (void *)e->off_words, (void *)e->off_exc, (void *)e->totals, (void *)e->packed,
                  (void *)e->exc, (void *)e->pos, (void *)e->f32_sizes, (void *)e->f32_offs,
                  (void *)e->f32_blk, (void *)e->f32_tot})
    if (p) cudaFree(p);
  e->f32_sizes = nullptr;
  e->f32_offs = e->f32_blk = e->f32_tot = nullptr;
  e->feat = nullptr;
  e->labels = e->cand = nullptr;
  e->sl = EncodeSlots{};
  e->off_words = e->off_exc = e->totals = nullptr;
  e->packed = nullptr;
  e->exc = nullptr;
  e->pos = nullptr;
  e->cap_vecs = 0;
}

flsgpu_status ensure_vecs(flsgpu_alp_encoder *e, size_t n_vecs) {
  if (n_vecs <= e->cap_vecs) return FLSGPU_OK;
  free_enc(e);
  flsgpu_status st = FLSGPU_OK;
  const size_t n = n_vecs;
  e->feat = dalloc<bf16>(n * kFeatures, st);
  e->labels = dalloc<int16_t>(n, st);
  e->cand = dalloc<int16_t>(n * 4, st);
  e->sl.fill = dalloc<int64_t>(n, st);
  e->sl.fb_list = dalloc<uint32_t>(n, st);
  e->sl.fb_count = dalloc<uint32_t>(1, st);
  e->sl.blk_words = dalloc<size_t>(n / 1024 + 1, st);
  e->sl.blk_exc = dalloc<size_t>(n / 1024 + 1, st);
  e->sl.exc_mask = dalloc<uint32_t>(n * 32, st);
  e->sl.bw = dalloc<uint8_t>(n, st);
  e->sl.base = dalloc<uint64_t>(n, st);
  e->sl.fac = dalloc<uint8_t>(n, st);
  e->sl.exp = dalloc<uint8_t>(n, st);
  e->sl.count = dalloc<uint16_t>(n, st);
  e->sl.flags = dalloc<uint8_t>(n, st);
  e->off_words = dalloc<size_t>(n, st);
  e->off_exc = dalloc<size_t>(n, st);
  e->totals = dalloc<size_t>(8, st);
  e->packed = dalloc<uint64_t>(n * VEC, st);
  e->exc = dalloc<double>(n * VEC, st);
  e->pos = dalloc<uint16_t>(n * VEC, st);
  e->f32_sizes = dalloc<uint32_t>(2 * n, st);
  e->f32_offs = dalloc<size_t>(2 * n, st);
  e->f32_blk = dalloc<size_t>(2 * (n / 1024 + 1), st);
  e->f32_tot = dalloc<size_t>(4, st);
  if (st == FLSGPU_OK) e->cap_vecs = n;
  return st;
}

flsgpu_status refresh_bf16(flsgpu_alp_encoder *e, cudaStream_t s) {
  k_to_bf16<<<(kW1 + 255) / 256, 256, 0, s>>>(e->w + kOffW1, kW1, e->w1b, nullptr, kHidden, kFeatures);
  k_to_bf16<<<(kW2 + 255) / 256, 256, 0, s>>>(e->w + kOffW2, kW2, e->w2b, e->w2t, kHidden, kHidden);
  k_to_bf16<<<(kW3 + 255) / 256, 256, 0, s>>>(e->w + kOffW3, kW3, e->w3b, e->w3t, kOut, kHidden);
  note_launch(3);
  return check_cuda(cudaGetLastError(), "refresh weights");
}

GemmArgs gemm(const bf16 *A, int lda, const bf16 *B, int ldb, int M, int N, int K, float *Cf,
              bf16 *Cb, int ldc, const float *bias, int relu, uint32_t *status) {
  return GemmArgs{A, B, lda, ldb, M, N, K, Cf, Cb, ldc, bias, relu, status};
}

// forward of `rows` feature rows already in e->x: h1, h2 (bf16), z (fp32)
flsgpu_status forward(flsgpu_alp_encoder *e, const bf16 *x, int rows, cudaStream_t s) {
  flsgpu_status st;
  if ((st = gemm_tn(gemm(x, kFeatures, e->w1b, kFeatures, rows, kHidden, kFeatures, nullptr, e->h1,
                         kHidden, e->w + kOffB1, 1, e->status), s)))
    return st;
  if ((st = gemm_tn(gemm(e->h1, kHidden, e->w2b, kHidden, rows, kHidden, kHidden, nullptr, e->h2,
                         kHidden, e->w + kOffB2, 1, e->status), s)))
    return st;
  return gemm_tn(gemm(e->h2, kHidden, e->w3b, kHidden, rows, kOut, kHidden, e->z, nullptr, kOut,
                      e->w + kOffB3, 0, e->status), s);
}

void transpose(const bf16 *in, int rows, int cols, bf16 *out, int ld_out, cudaStream_t s) {
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  k_transpose_bf16<<<grid, block, 0, s>>>(in, rows, cols, cols, out, ld_out);
  note_launch();
}

// forward + backward of one batch (rows % 16 == 0): gradients into e->g,
// per-row losses into e->loss
flsgpu_status forward_backward(flsgpu_alp_encoder *e, const bf16 *x, const int16_t *labels,
                               int rows, cudaStream_t s) {
  flsgpu_status st;
  if ((st = forward(e, x, rows, s))) return st;
  const int wb = (rows * 32 + 255) / 256;
  k_softmax_ce<<<wb, 256, 0, s>>>(e->z, labels, rows, e->loss, e->dz);
  note_launch();
  // layer 3: dW3 = dZ^T H2 ; db3 = colsum dZ ; dH2 = dZ W3
  transpose(e->dz, rows, kOut, e->t_a, rows, s);     // dZ^T [192 x rows]
  transpose(e->h2, rows, kHidden, e->t_b, rows, s);  // H2^T [128 x rows]
  if ((st = gemm_tn(gemm(e->t_a, rows, e->t_b, rows, kOut, kHidden, rows, e->g + kOffW3, nullptr,
                         kHidden, nullptr, 0, e->status), s)))
    return st;
  k_colsum_bf16<<<(kOut + 31) / 32, dim3(32, 32), 0, s>>>(e->dz, rows, kOut, e->g + kOffB3);
  if ((st = gemm_tn(gemm(e->dz, kOut, e->w3t, kOut, rows, kHidden, kOut, e->tmpf, nullptr, kHidden,
                         nullptr, 0, e->status), s)))
    return st;
  k_relu_back<<<592, 256, 0, s>>>(e->tmpf, e->h2, rows, kHidden, e->dh);
  // layer 2: dW2 = dH2^T H1 ; db2 ; dH1 = dH2 W2
  transpose(e->dh, rows, kHidden, e->t_a, rows, s);
  transpose(e->h1, rows, kHidden, e->t_b, rows, s);
  if ((st = gemm_tn(gemm(e->t_a, rows, e->t_b, rows, kHidden, kHidden, rows, e->g + kOffW2, nullptr,
                         kHidden, nullptr, 0, e->status), s)))
    return st;
  k_colsum_bf16<<<(kHidden + 31) / 32, dim3(32, 32), 0, s>>>(e->dh, rows, kHidden, e->g + kOffB2);
  if ((st = gemm_tn(gemm(e->dh, kHidden, e->w2t, kHidden, rows, kHidden, kHidden, e->tmpf, nullptr,
                         kHidden, nullptr, 0, e->status), s)))
    return st;
  k_relu_back<<<592, 256, 0, s>>>(e->tmpf, e->h1, rows, kHidden, e->dh);
  // layer 1: dW1 = dH1^T X ; db1
  transpose(e->dh, rows, kHidden, e->t_a, rows, s);
  transpose(x, rows, kFeatures, e->t_b, rows, s);
  if ((st = gemm_tn(gemm(e->t_a, rows, e->t_b, rows, kHidden, kFeatures, rows, e->g + kOffW1,
                         nullptr, kFeatures, nullptr, 0, e->status), s)))
    return st;
  k_colsum_bf16<<<(kHidden + 31) / 32, dim3(32, 32), 0, s>>>(e->dh, rows, kHidden, e->g + kOffB1);
  note_launch(5);
  return check_cuda(cudaGetLastError(), "backward");
}

flsgpu_status adam_step(flsgpu_alp_encoder *e, float lr, cudaStream_t s) {
  e->adam_t++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)e->adam_t), c2 = 1.0f - powf(b2, (float)e->adam_t);
  struct P {
    int off, n, rows, cols;
    bf16 *wb, *wt;
  } ps[6] = {{kOffW1, kW1, kHidden, kFeatures, e->w1b, nullptr}, {kOffB1, kB1, 1, kB1, nullptr, nullptr},
             {kOffW2, kW2, kHidden, kHidden, e->w2b, e->w2t},     {kOffB2, kB2, 1, kB2, nullptr, nullptr},
             {kOffW3, kW3, kOut, kHidden, e->w3b, e->w3t},        {kOffB3, kB3, 1, kB3, nullptr, nullptr}};
  for (const P &p : ps) {
    k_adam<<<(p.n + 255) / 256, 256, 0, s>>>(e->w + p.off, e->g + p.off, e->m + p.off, e->v + p.off,
                                             p.n, lr, b1, b2, 1e-8f, c1, c2, p.wb, p.wt, p.rows, p.cols);
  }
  note_launch(6);
  return check_cuda(cudaGetLastError(), "adam");
}

flsgpu_status features(const double *vals, size_t n_vecs, bf16 *feat, cudaStream_t s) {
  if (!n_vecs) return FLSGPU_OK;
  k_features<<<persistent_blocks(n_vecs, 8, 4), 256, 0, s>>>(vals, n_vecs, feat);
  note_launch();
  return check_cuda(cudaGetLastError(), "k_features");
}

// The proposals in one fused launch (k_propose).
flsgpu_status propose(flsgpu_alp_encoder *e, const double *vals, size_t n_vecs, int k,
                      cudaStream_t s) {
  if (!n_vecs) return FLSGPU_OK;
  static bool attr = false;
  if (!attr) {
    flsgpu_status st = check_cuda(
        cudaFuncSetAttribute(k_propose, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPropSmem),
        "k_propose attribute");
    if (st) return st;
    attr = true;
  }
  const size_t tiles = (n_vecs + kPropRows - 1) / kPropRows;
  const unsigned grid =
      (unsigned)std::min<size_t>((tiles + kPropTeams - 1) / kPropTeams, (size_t)sm_count());
  k_propose<<<grid, kPropThreads, kPropSmem, s>>>(vals, n_vecs, e->w1b, e->w2b, e->w3b, e->w + kOffB1,
                                               e->w + kOffB2, e->w + kOffB3, k, e->cand, e->status);
  note_launch();
  return check_cuda(cudaGetLastError(), "k_propose launch");
}

// The same proposals layer by layer: features, three GEMM launches, top-k.
flsgpu_status propose_layered(flsgpu_alp_encoder *e, const double *vals, size_t n_vecs, int k,
                              cudaStream_t s) {
  flsgpu_status st;
  if ((st = features(vals, n_vecs, e->feat, s))) return st;
  const int chunk = 1 << 16;
  if ((st = ensure_rows(e, (int)std::min<size_t>(n_vecs, chunk)))) return st;
  for (size_t r0 = 0; r0 < n_vecs; r0 += chunk) {
    const int rows = (int)std::min<size_t>(chunk, n_vecs - r0);
    if ((st = forward(e, e->feat + r0 * kFeatures, rows, s))) return st;
    k_topk<<<(rows * 32 + 255) / 256, 256, 0, s>>>(e->z, rows, k, e->cand + r0 * k);
    note_launch();
  }
  return check_cuda(cudaGetLastError(), "propose");
}

}  // namespace

namespace flsb200 {

template <typename T>
static flsgpu_status alprd_encode(flsgpu_alp_encoder *e, const T *d_values, size_t n_values,
                                  uint32_t rowgroup_vecs, flsgpu_alprd_encode_result *out,
                                  flsgpu_stream stream) {
  if (!e || !d_values || !out || (n_values % VEC) || rowgroup_vecs < 1 || rowgroup_vecs > 100)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT,
                     "ALP-RD encode: null argument, n_values not a multiple of 1024, or "
                     "rowgroup_vecs outside 1..100");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t n_vecs = n_values / VEC;
  flsgpu_status st = rd_work_reserve(e->rd, n_vecs);
  if (st) return st;
  if ((st = run_rd_encode<T>(d_values, n_vecs, (int)rowgroup_vecs, e->rd, s))) return st;
  size_t tot[3] = {0, 0, 0};
  if (n_vecs &&
      ((st = check_cuda(cudaMemcpyAsync(tot, e->rd.totals, sizeof(tot), cudaMemcpyDeviceToHost, s),
                        "copy")) ||
       (st = check_cuda(cudaStreamSynchronize(s), "sync"))))
    return st;
  std::memset(out, 0, sizeof(*out));
  flsgpu_alprd_column &c = out->column;
  RDWork &w = e->rd;
  c.n_values = n_values;
  c.right = flsgpu_bp_column{n_values, n_vecs, w.right, w.rbw, w.offs};
  c.left = flsgpu_bp_column{n_values, n_vecs, w.left, w.lbw, w.offs + w.cap};
  c.dictionaries = w.dicts;
  c.dictionary_indices = w.dict_idx;
  c.n_exceptions = tot[2];
  c.exceptions_offsets = w.offs + 2 * w.cap;
  c.exceptions = w.exc;
  c.positions = w.pos;
  c.counts = w.count;
  const size_t n_dict = (n_vecs + rowgroup_vecs - 1) / rowgroup_vecs;
  out->n_right_words = tot[0];
  out->n_left_words = tot[1];
  out->n_exceptions = tot[2];
  out->n_dictionaries = n_dict;
  // packed words, 4 B per exception (left part + position), 16 B per
  // dictionary, and per vector the two widths, three offsets, the
  // dictionary index and the exception count (32 B)
  out->compressed_bytes = tot[0] * sizeof(T) + tot[1] * 2 + tot[2] * 4 + n_dict * 16 + n_vecs * 32;
  return FLSGPU_OK;
}

}  // namespace flsb200

extern "C" {

flsgpu_status flsgpu_alp_encoder_create(uint32_t seed, flsgpu_alp_encoder **out) {
  if (!out) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null output");
  auto *e = new flsgpu_alp_encoder();
  flsgpu_status st = FLSGPU_OK;
  e->w = dalloc<float>(kParams, st);
  e->m = dalloc<float>(kParams, st);
  e->v = dalloc<float>(kParams, st);
  e->g = dalloc<float>(kParams, st);
  e->w1b = dalloc<bf16>(kW1, st);
  e->w2b = dalloc<bf16>(kW2, st);
  e->w3b = dalloc<bf16>(kW3, st);
  e->w2t = dalloc<bf16>(kW2, st);
  e->w3t = dalloc<bf16>(kW3, st);
  e->status = dalloc<uint32_t>(1, st);
  if (st == FLSGPU_OK) {
    // He-uniform initialisation, zero biases; the padding class gets a
    // large negative bias so it is never proposed
    std::vector<float> h(kParams, 0.0f);
    std::mt19937 rng(seed);
    auto fill = [&](int off, int n, int fan_in) {
      std::uniform_real_distribution<float> d(-std::sqrt(6.0f / fan_in), std::sqrt(6.0f / fan_in));
      for (int i = 0; i < n; ++i) h[off + i] = d(rng);
    };
    fill(kOffW1, kW1, kFeatures);
    fill(kOffW2, kW2, kHidden);
    fill(kOffW3, kW3, kHidden);
    for (int c = 0; c < kHidden; ++c) h[kOffW3 + (kOut - 1) * kHidden + c] = 0.0f;
    h[kOffB3 + kOut - 1] = -30.0f;
    st = check_cuda(cudaMemcpy(e->w, h.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice), "copy");
    if (!st) st = check_cuda(cudaMemset(e->m, 0, sizeof(float) * kParams), "memset");
    if (!st) st = check_cuda(cudaMemset(e->v, 0, sizeof(float) * kParams), "memset");
    if (!st) st = check_cuda(cudaMemset(e->status, 0, 4), "memset");
    if (!st) st = refresh_bf16(e, nullptr);
    if (!st) st = check_cuda(cudaDeviceSynchronize(), "sync");
  }
  if (st) {
    flsgpu_alp_encoder_destroy(e);
    return st;
  }
  *out = e;
  return FLSGPU_OK;
}

void flsgpu_alp_encoder_destroy(flsgpu_alp_encoder *e) {
  if (!e) return;
  free_acts(e);
  free_enc(e);
  rd_work_free(e->rd);
  for (void *p : {(void *)e->w, (void *)e->m, (void *)e->v, (void *)e->g, (void *)e->w1b,
                  (void *)e->w2b, (void *)e->w3b, (void *)e->w2t, (void *)e->w3t, (void *)e->status})
    if (p) cudaFree(p);
  delete e;
}

size_t flsgpu_alp_encoder_param_count(void) { return kParams; }

flsgpu_status flsgpu_alp_encoder_get_params(const flsgpu_alp_encoder *e, float *h_params) {
  if (!e || !h_params) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null argument");
  return check_cuda(cudaMemcpy(h_params, e->w, sizeof(float) * kParams, cudaMemcpyDeviceToHost), "copy");
}

flsgpu_status flsgpu_alp_encoder_set_params(flsgpu_alp_encoder *e, const float *h_params) {
  if (!e || !h_params) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null argument");
  flsgpu_status st =
      check_cuda(cudaMemcpy(e->w, h_params, sizeof(float) * kParams, cudaMemcpyHostToDevice), "copy");
  if (!st) st = refresh_bf16(e, nullptr);
  if (!st) st = check_cuda(cudaDeviceSynchronize(), "sync");
  return st;
}

// Gradients of the mean cross entropy of `rows` labelled feature rows
// (d_features: rows x 64 bf16) with respect to every parameter, written to
// d_grads (flsgpu_alp_encoder_param_count() floats, the parameter layout);
// *h_loss receives the mean loss.  Synchronises.
flsgpu_status flsgpu_alp_encoder_gradients(flsgpu_alp_encoder *e, const void *d_features,
                                           const int16_t *d_labels, uint32_t rows, float *d_grads,
                                           float *h_loss, flsgpu_stream stream) {
  if (!e || !d_features || !d_labels || !rows || (rows % 16))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "gradients: rows must be a positive multiple of 16");
  cudaStream_t s = (cudaStream_t)stream;
  flsgpu_status st = ensure_rows(e, (int)rows);
  if (!st) st = forward_backward(e, static_cast<const bf16 *>(d_features), d_labels, (int)rows, s);
  if (!st && d_grads)
    st = check_cuda(cudaMemcpyAsync(d_grads, e->g, sizeof(float) * kParams, cudaMemcpyDeviceToDevice, s), "copy");
  if (!st) st = check_cuda(cudaStreamSynchronize(s), "sync");
  if (!st && h_loss) {
    std::vector<float> l(rows);
    st = check_cuda(cudaMemcpy(l.data(), e->loss, sizeof(float) * rows, cudaMemcpyDeviceToHost), "copy");
    double acc = 0;
    for (float x : l) acc += x;
    *h_loss = (float)(acc / rows);
  }
  return st;
}

flsgpu_status flsgpu_alp_features(const double *d_values, size_t n_values, void *d_features,
                                  flsgpu_stream stream) {
  if (n_values % VEC) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "n_values must be a multiple of 1024");
  return features(d_values, n_values / VEC, static_cast<bf16 *>(d_features), (cudaStream_t)stream);
}

flsgpu_status flsgpu_alp_plain_labels(const double *d_values, size_t n_values, int16_t *d_labels,
                                      int32_t *d_est, flsgpu_stream stream) {
  if (n_values % VEC) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "n_values must be a multiple of 1024");
  return run_plain_labels(d_values, n_values / VEC, d_labels, d_est, (cudaStream_t)stream);
}

// Trains the network on the plain search's labels of `d_values` (features
// and labels computed on the GPU), `epochs` passes of Adam over shuffled
// minibatches of `batch` rows.  Synchronises; reports the mean loss of the
// first and the last epoch.
flsgpu_status flsgpu_alp_encoder_train(flsgpu_alp_encoder *e, const double *d_values,
                                       size_t n_values, uint32_t epochs, uint32_t batch, float lr,
                                       float *h_loss_first, float *h_loss_last,
                                       flsgpu_stream stream) {
  if (!e || !d_values || (n_values % VEC) || !batch || (batch % 128))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "train: n_values % 1024 and batch % 128 must be 0");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t n_vecs = n_values / VEC;
  flsgpu_status st = ensure_vecs(e, n_vecs);
  if (!st) st = ensure_rows(e, (int)batch);
  if (!st) st = features(d_values, n_vecs, e->feat, s);
  if (!st) st = run_plain_labels(d_values, n_vecs, e->labels, nullptr, s);
  if (st) return st;
  // every epoch visits the rows in a new order: a keyed permutation of the
  // row indices, gathered into a batch-ordered copy on the device
  const size_t nb = n_vecs / batch;
  if (nb == 0) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "fewer vectors than one batch");
  bf16 *dfeat = nullptr;
  int16_t *dlab = nullptr;
  st = check_cuda(cudaMalloc(&dfeat, sizeof(bf16) * nb * batch * kFeatures), "cudaMalloc");
  if (!st) st = check_cuda(cudaMalloc(&dlab, sizeof(int16_t) * nb * batch), "cudaMalloc");
  int half_bits = 1;
  while ((1ull << (2 * half_bits)) < n_vecs) ++half_bits;
  std::vector<float> lbuf(batch);
  for (uint32_t ep = 0; ep < epochs && !st; ++ep) {
    const uint32_t key = 0x9E3779B9u * (ep + 1) ^ 1234u;
    const size_t rows = nb * batch;
    k_gather_rows<<<(unsigned)((rows * 8 + 255) / 256), 256, 0, s>>>(
        e->feat, e->labels, (uint32_t)n_vecs, rows, half_bits, key, dfeat, dlab);
    note_launch();
    st = check_cuda(cudaGetLastError(), "k_gather_rows");
    double eloss = 0;
    for (size_t b = 0; b < nb && !st; ++b) {
      st = forward_backward(e, dfeat + b * batch * kFeatures, dlab + b * batch, (int)batch, s);
      if (!st) st = adam_step(e, lr, s);
      if (!st && (ep == 0 || ep + 1 == epochs)) {
        st = check_cuda(cudaMemcpyAsync(lbuf.data(), e->loss, sizeof(float) * batch, cudaMemcpyDeviceToHost, s), "copy");
        if (!st) st = check_cuda(cudaStreamSynchronize(s), "sync");
        for (float x : lbuf) eloss += x;
      }
    }
    if (!st && ep == 0 && h_loss_first) *h_loss_first = (float)(eloss / (nb * batch));
    if (!st && ep + 1 == epochs && h_loss_last) *h_loss_last = (float)(eloss / (nb * batch));
  }
  if (!st) st = check_cuda(cudaStreamSynchronize(s), "sync");
  cudaFree(dfeat);
  cudaFree(dlab);
  uint32_t hst = 0;
  if (!st) cudaMemcpy(&hst, e->status, 4, cudaMemcpyDeviceToHost);
  if (!st && hst) st = set_error(FLSGPU_ERR_TIMEOUT, "tensor-core wait gave up (status %x)", hst);
  return st;
}

// Top-k (k <= 4) proposed classes per vector (d_cand: n_vecs x k int16).
flsgpu_status flsgpu_alp_encoder_propose(flsgpu_alp_encoder *e, const double *d_values,
                                         size_t n_values, uint32_t k, int16_t *d_cand,
                                         flsgpu_stream stream) {
  if (!e || !d_values || (n_values % VEC) || k < 1 || k > 4)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "propose: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t n_vecs = n_values / VEC;
  flsgpu_status st = ensure_vecs(e, n_vecs);
  if (!st) st = propose(e, d_values, n_vecs, (int)k, s);
  if (!st && d_cand)
    st = check_cuda(cudaMemcpyAsync(d_cand, e->cand, sizeof(int16_t) * n_vecs * k, cudaMemcpyDeviceToDevice, s), "copy");
  return st;
}

// The layer-by-layer path of the same proposals (features, three GEMM
// launches, top-k): kept so that tests can hold the fused kernel to it.
flsgpu_status flsgpu_alp_encoder_propose_layered(flsgpu_alp_encoder *e, const double *d_values,
                                                 size_t n_values, uint32_t k, int16_t *d_cand,
                                                 flsgpu_stream stream) {
  if (!e || !d_values || (n_values % VEC) || k < 1 || k > 4)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "propose: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t n_vecs = n_values / VEC;
  flsgpu_status st = ensure_vecs(e, n_vecs);
  if (!st) st = propose_layered(e, d_values, n_vecs, (int)k, s);
  if (!st && d_cand)
    st = check_cuda(cudaMemcpyAsync(d_cand, e->cand, sizeof(int16_t) * n_vecs * k, cudaMemcpyDeviceToDevice, s), "copy");
  return st;
}

flsgpu_status flsgpu_alp_encoder_save(const flsgpu_alp_encoder *e, const char *path) {
  if (!e || !path) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<float> h(kParams);
  flsgpu_status st = flsgpu_alp_encoder_get_params(e, h.data());
  if (st) return st;
  FILE *f = fopen(path, "wb");
  if (!f) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "cannot open %s", path);
  const char magic[8] = {'F', 'L', 'S', 'A', 'L', 'P', 'N', '1'};
  const uint32_t dims[4] = {kFeatures, kHidden, kHidden, kOut};
  const bool ok = fwrite(magic, 1, 8, f) == 8 && fwrite(dims, 4, 4, f) == 4 &&
                  fwrite(h.data(), sizeof(float), kParams, f) == (size_t)kParams;
  fclose(f);
  return ok ? FLSGPU_OK : set_error(FLSGPU_ERR_INVALID_ARGUMENT, "short write to %s", path);
}

flsgpu_status flsgpu_alp_encoder_load(flsgpu_alp_encoder *e, const char *path) {
  if (!e || !path) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null argument");
  FILE *f = fopen(path, "rb");
  if (!f) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "cannot open %s", path);
  char magic[8];
  uint32_t dims[4];
  std::vector<float> h(kParams);
  const bool ok = fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "FLSALPN1", 8) == 0 &&
                  fread(dims, 4, 4, f) == 4 && dims[0] == kFeatures && dims[1] == kHidden &&
                  dims[2] == kHidden && dims[3] == kOut &&
                  fread(h.data(), sizeof(float), kParams, f) == (size_t)kParams;
  fclose(f);
  if (!ok) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "%s is not a proposal network file", path);
  return flsgpu_alp_encoder_set_params(e, h.data());
}

// Encodes an f64 column (n_values % 1024 == 0) into the reference's
// ALPColumn layout on the device.  mode 0: plain per-vector search;
// mode 1: the network's top-3 pairs, verified on the vector's samples, with
// the plain search as fallback above 3% exceptions.  The column's arrays
// live in the encoder's workspace until its next encode.  Synchronises to
// read the sizes.
flsgpu_status flsgpu_alp_encode_f64(flsgpu_alp_encoder *e, const double *d_values,
                                    size_t n_values, uint32_t mode,
                                    flsgpu_alp_encode_result *out, flsgpu_stream stream) {
  if (!e || !d_values || !out || (n_values % VEC) || mode > 1)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "encode: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t n_vecs = n_values / VEC;
  flsgpu_status st = ensure_vecs(e, n_vecs);
  if (st) return st;
  if (mode == 1 && (st = propose(e, d_values, n_vecs, 3, s))) return st;
  if ((st = run_alp_encode(d_values, n_vecs, (int)mode, e->cand, 3, 30, e->sl, e->off_words,
                           e->off_exc, e->totals, e->packed, e->exc, e->pos, s)))
    return st;
  size_t tot[5] = {0, 0, 0, 0, 0};
  if ((st = check_cuda(cudaMemcpyAsync(tot, e->totals, sizeof(tot), cudaMemcpyDeviceToHost, s), "copy")) ||
      (st = check_cuda(cudaStreamSynchronize(s), "sync")))
    return st;
  const size_t fb = tot[2], rd = tot[3], bwsum = tot[4];
  std::memset(out, 0, sizeof(*out));
  flsgpu_alp_column &c = out->column;
  c.n_values = n_values;
  c.ffor.n_values = n_values;
  c.ffor.bp.n_values = n_values;
  c.ffor.bp.n_vecs = n_vecs;
  c.ffor.bp.packed_array = e->packed;
  c.ffor.bp.bit_widths = e->sl.bw;
  c.ffor.bp.vector_offsets = e->off_words;
  c.ffor.bases = e->sl.base;
  c.factor_indices = e->sl.fac;
  c.fraction_indices = e->sl.exp;
  c.n_exceptions = tot[1];
  c.exceptions_offsets = e->off_exc;
  c.exceptions = e->exc;
  c.positions = e->pos;
  c.counts = e->sl.count;
  out->n_packed_words = tot[0];
  out->n_exceptions = tot[1];
  // reference accounting (alp-bindings.cu:19-43): packed bytes + 10 B per
  // exception + 3 + 8 B of per-vector overhead
  out->compressed_bytes = tot[0] * 8 + tot[1] * 10 + n_vecs * 11;
  out->n_fallback = fb;
  out->n_rd = rd;
  out->mean_bit_width = n_vecs ? (double)bwsum / (double)n_vecs : 0.0;
  return FLSGPU_OK;
}

flsgpu_status flsgpu_alprd_encode_f64(flsgpu_alp_encoder *e, const double *d_values,
                                      size_t n_values, uint32_t rowgroup_vecs,
                                      flsgpu_alprd_encode_result *out, flsgpu_stream stream) {
  return alprd_encode<double>(e, d_values, n_values, rowgroup_vecs, out, stream);
}

flsgpu_status flsgpu_alprd_encode_f32(flsgpu_alp_encoder *e, const float *d_values,
                                      size_t n_values, uint32_t rowgroup_vecs,
                                      flsgpu_alprd_encode_result *out, flsgpu_stream stream) {
  return alprd_encode<float>(e, d_values, n_values, rowgroup_vecs, out, stream);
}

flsgpu_status flsgpu_alp_encode_hybrid_f64(flsgpu_alp_encoder *e, const double *d_values,
                                           size_t n_values, uint32_t mode,
                                           flsgpu_alp_hybrid_encode_result *out,
                                           flsgpu_stream stream) {
  if (!e || !d_values || !out || (n_values % VEC) || mode > 1)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "hybrid encode: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t n_vecs = n_values / VEC;
  flsgpu_status st = ensure_vecs(e, n_vecs);
  if (st || (st = rd_work_reserve(e->rd, n_vecs))) return st;
  if (mode == 1 && (st = propose(e, d_values, n_vecs, 3, s))) return st;
  if ((st = run_alp_encode(d_values, n_vecs, (int)mode, e->cand, 3, 30, e->sl, e->off_words,
                           e->off_exc, e->totals, e->packed, e->exc, e->pos, s, &e->rd)))
    return st;
  size_t tot[5] = {0, 0, 0, 0, 0}, rtot[3] = {0, 0, 0};
  if ((st = check_cuda(cudaMemcpyAsync(tot, e->totals, sizeof(tot), cudaMemcpyDeviceToHost, s), "copy")) ||
      (st = check_cuda(cudaMemcpyAsync(rtot, e->rd.totals, sizeof(rtot), cudaMemcpyDeviceToHost, s),
                       "copy")) ||
      (st = check_cuda(cudaStreamSynchronize(s), "sync")))
    return st;
  std::memset(out, 0, sizeof(*out));
  flsgpu_alphybrid_column &h = out->column;
  h.n_values = n_values;
  flsgpu_alp_column &c = h.alp;
  c.n_values = n_values;
  c.ffor.n_values = n_values;
  c.ffor.bp.n_values = n_values;
  c.ffor.bp.n_vecs = n_vecs;
  c.ffor.bp.packed_array = e->packed;
  c.ffor.bp.bit_widths = e->sl.bw;
  c.ffor.bp.vector_offsets = e->off_words;
  c.ffor.bases = e->sl.base;
  c.factor_indices = e->sl.fac;
  c.fraction_indices = e->sl.exp;
  c.n_exceptions = tot[1];
  c.exceptions_offsets = e->off_exc;
  c.exceptions = e->exc;
  c.positions = e->pos;
  c.counts = e->sl.count;
  RDWork &w = e->rd;
  flsgpu_alprd_column &r = h.rd;
  r.n_values = n_values;
  r.right = flsgpu_bp_column{n_values, n_vecs, w.right, w.rbw, w.offs};
  r.left = flsgpu_bp_column{n_values, n_vecs, w.left, w.lbw, w.offs + w.cap};
  r.dictionaries = w.dicts;
  r.dictionary_indices = w.dict_idx;
  r.n_exceptions = rtot[2];
  r.exceptions_offsets = w.offs + 2 * w.cap;
  r.exceptions = w.exc;
  r.positions = w.pos;
  r.counts = w.count;
  h.schemes = w.scheme;
  const size_t n_rd = tot[3], n_alp = n_vecs - n_rd;
  out->n_alp_vectors = n_alp;
  out->n_rd_vectors = n_rd;
  out->n_packed_words = tot[0];
  out->n_exceptions = tot[1];
  out->n_right_words = rtot[0];
  out->n_left_words = rtot[1];
  out->n_rd_exceptions = rtot[2];
  out->n_fallback = tot[2];
  out->mean_bit_width = n_alp ? (double)tot[4] / (double)n_alp : 0.0;
  out->d_flags = e->sl.flags;
  // ALP vectors as alp::encode accounts them (alp-bindings.cu:19-43: packed
  // bytes, 10 B per exception, 11 B per vector); ALP-RD vectors: packed
  // words, 4 B per exception, a 16 B dictionary and 32 B of metadata; one
  // scheme byte per vector
  out->compressed_bytes = tot[0] * 8 + tot[1] * 10 + n_alp * 11 + rtot[0] * 8 + rtot[1] * 2 +
                          rtot[2] * 4 + n_rd * 48 + n_vecs;
  return FLSGPU_OK;
}

flsgpu_status flsgpu_alp_encode_f32(flsgpu_alp_encoder *e, const float *d_values,
                                    size_t n_values, flsgpu_alp_encode_result *out,
                                    flsgpu_stream stream) {
  if (!e || !d_values || !out || (n_values % VEC))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "f32 encode: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t n_vecs = n_values / VEC;
  flsgpu_status st = ensure_vecs(e, n_vecs);
  if (st) return st;
  const size_t stride = e->cap_vecs, bstride = e->cap_vecs / 1024 + 1;
  Enc32Slots sl{};
  sl.bw = e->sl.bw;
  sl.fac = e->sl.fac;
  sl.exp = e->sl.exp;
  sl.base = reinterpret_cast<uint32_t *>(e->sl.base);
  sl.fill = reinterpret_cast<int32_t *>(e->sl.fill);
  sl.count = e->sl.count;
  sl.exc_mask = e->sl.exc_mask;
  sl.sizes = e->f32_sizes;
  sl.stride = stride;
  sl.n_rd = e->f32_tot + 2;
  uint32_t *packed = reinterpret_cast<uint32_t *>(e->packed);
  float *exc = reinterpret_cast<float *>(e->exc);
  size_t tot[3] = {0, 0, 0};
  if (n_vecs &&
      ((st = check_cuda(cudaMemsetAsync(e->f32_tot + 2, 0, sizeof(size_t), s), "memset")) ||
       (st = run_alp_encode_f32(d_values, n_vecs, sl, e->f32_offs, e->f32_blk, bstride,
                                e->f32_tot, packed, exc, e->pos, s)) ||
       (st = check_cuda(cudaMemcpyAsync(tot, e->f32_tot, sizeof(tot), cudaMemcpyDeviceToHost, s),
                        "copy")) ||
       (st = check_cuda(cudaStreamSynchronize(s), "sync"))))
    return st;
  std::memset(out, 0, sizeof(*out));
  flsgpu_alp_column &c = out->column;
  c.n_values = n_values;
  c.ffor.n_values = n_values;
  c.ffor.bp.n_values = n_values;
  c.ffor.bp.n_vecs = n_vecs;
  c.ffor.bp.packed_array = packed;
  c.ffor.bp.bit_widths = sl.bw;
  c.ffor.bp.vector_offsets = e->f32_offs;
  c.ffor.bases = sl.base;
  c.factor_indices = sl.fac;
  c.fraction_indices = sl.exp;
  c.n_exceptions = tot[1];
  c.exceptions_offsets = e->f32_offs + stride;
  c.exceptions = exc;
  c.positions = e->pos;
  c.counts = sl.count;
  out->n_packed_words = tot[0];
  out->n_exceptions = tot[1];
  // reference accounting (alp-bindings.cu:19-43): packed bytes, 6 B per
  // exception (value + position), 3 + 4 B of per-vector metadata
  out->compressed_bytes = tot[0] * 4 + tot[1] * 6 + n_vecs * 7;
  out->n_fallback = 0;
  out->n_rd = tot[2];
  out->mean_bit_width = 0.0;
  return FLSGPU_OK;
}

}  // extern "C"
