// alp_encode.cu -- GPU ALP encoder for f64 columns: per-vector parameter
// search (plain, or proposed by the learned network and verified), encode
// with exceptions, FFOR analysis and FastLanes packing, then compaction
// into the reference's ALPColumn layout.
//
// The arithmetic restates the reference's CPU encoder:
//   encode_value  src/alp/encoder.hpp:77-84  (v * 10^e * 10^-f + M - M, cast)
//   decode_value  src/alp/decoder.hpp:124-127
//   sampling search over the 32 samples of a vector (every 32nd value, the
//     second-level sample of encoder.hpp:248-270) with the estimate and tie
//     rules of find_top_k_combinations, encoder.hpp:134-230
//   choice among candidates: find_best_exponent_factor_from_combinations,
//     encoder.hpp:237-300 (early exit after two non-improving candidates)
//   encode_simdized, encoder.hpp:302-379 (specials, exceptions, fill value)
//   analyze_ffor, encoder.hpp:104-115, and fls::ffor
// Conversions reproduce the x86 results of the reference's casts
// (out-of-range double -> int64 gives INT64_MIN), and every multiply and
// add is a separately rounded __dmul_rn / __dadd_rn (no contraction).
#include <cuda_bf16.h>

#include <cstring>
#include <vector>

#include "alp_learn.cuh"
#include "rd_encode.cuh"

namespace flsb200 {

static __constant__ double c_f64_exp10[19] = {1.0,  10.0, 100.0, 1e3,  1e4,  1e5,  1e6,
                                              1e7,  1e8,  1e9,   1e10, 1e11, 1e12, 1e13,
                                              1e14, 1e15, 1e16,  1e17, 1e18};

constexpr double kEncUpper = 9223372036854774784.0;  // constants.hpp:18
constexpr double kEncLower = -9223372036854774784.0;
constexpr double kMagic = 6755399441055744.0;         // 0x0018000000000000
// RD_SIZE_THRESHOLD_LIMIT (constants.hpp): 48 bits per value over the 32
// samples; a best estimate at or above it sends the data to ALP-RD
// (encoder.hpp:208-211)
constexpr int kRDLimitBits = 48 * 32;

__device__ __forceinline__ int64_t cvtt_s64(double x) {
  if (!(x >= -9223372036854775808.0 && x < 9223372036854775808.0)) return INT64_MIN;
  return (int64_t)x;
}

__device__ __forceinline__ bool impossible_f64(double n) {
  return !isfinite(n) || n > kEncUpper || n < kEncLower || (n == 0.0 && signbit(n));
}

__device__ __forceinline__ int64_t enc_value(double v, int f, int e, bool safe) {
  const double t = __dmul_rn(__dmul_rn(v, c_f64_exp10[e]), c_f64_frac[f]);
  if (safe && impossible_f64(t)) return (int64_t)kEncUpper;
  return cvtt_s64(__dsub_rn(__dadd_rn(t, kMagic), kMagic));
}

__device__ __forceinline__ double dec_value(int64_t q, int f, int e) {
  return __dmul_rn(__ll2double_rn((long long)((uint64_t)q * (uint64_t)c_f64_fact[f])),
                   c_f64_frac[e]);
}

// The stored integer of a non-exception value: the reference's
// round-to-integer by adding and subtracting 2^52 + 2^51.  For |t| < 2^51
// the sum lies in [2^52, 2^53), where its mantissa bits are the integer +
// 2^51, so the integer is read from the bits (no conversion instruction);
// larger magnitudes take the conversion.
__device__ __forceinline__ int64_t enc_stored(double x, double m10e, double mfrf) {
  const double t = __dmul_rn(__dmul_rn(x, m10e), mfrf);
  const double s = __dadd_rn(t, kMagic);
  if (fabs(t) < 2251799813685248.0)
    return (int64_t)((uint64_t)__double_as_longlong(s) & 0xFFFFFFFFFFFFFull) - 2251799813685248ll;
  return cvtt_s64(__dsub_rn(s, kMagic));
}

// dec_value with the factor and 10^-e in registers: the wrapped product
// q * 10^f converted to double through the magic sum when it lies in
// (-2^51, 2^51) (exact there), by the conversion otherwise.
__device__ __forceinline__ double dec_stored(int64_t q, uint64_t fact, double frce) {
  const uint64_t n = (uint64_t)q * fact;
  const double dn =
      n + 2251799813685248ull < 4503599627370496ull
          ? __dsub_rn(__longlong_as_double((long long)(n + 0x4338000000000000ull)), kMagic)
          : __ll2double_rn((long long)n);
  return __dmul_rn(dn, frce);
}

__device__ __forceinline__ int count_bits64(uint64_t x) { return x ? 64 - __clzll((long long)x) : 0; }

__device__ __forceinline__ int64_t warp_max_s64(int64_t x) {
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const int64_t y = __shfl_xor_sync(0xffffffffu, x, s);
    x = y > x ? y : x;
  }
  return x;
}
__device__ __forceinline__ int64_t warp_min_s64(int64_t x) {
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const int64_t y = __shfl_xor_sync(0xffffffffu, x, s);
    x = y < x ? y : x;
  }
  return x;
}

// Estimated sample bits of pair (e, f) over the warp's 32 samples (lane i
// holds sample i) with the sampling search's formula; -1 when fewer than two
// samples round-trip (find_top_k_combinations skips the pair).
__device__ __forceinline__ int sample_estimate(double s, int e, int f, bool skip_few) {
  const int64_t enc = enc_value(s, f, e, true);
  const bool ok = dec_value(enc, f, e) == s;
  const unsigned m = __ballot_sync(0xffffffffu, ok);
  const int nonexc = __popc(m);
  if (skip_few && nonexc < 2) return -1;
  const int64_t mx = warp_max_s64(ok ? enc : INT64_MIN);
  const int64_t mn = warp_min_s64(ok ? enc : INT64_MAX);
  const int bits = count_bits64((uint64_t)mx - (uint64_t)mn);
  return 32 * bits + (32 - nonexc) * (64 + 16);
}

// Exhaustive search over the 190 pairs (0 <= f <= e <= 18) on the warp's
// 32 samples (smp, shared memory), with the estimate and tie rules of
// find_top_k_combinations.  Lane l evaluates the pairs of class l, l + 32,
// ... over all samples, so no per-pair warp reduction is needed; a single
// warp minimum over (estimate, 18 - e, 18 - f) then picks the pair the
// reference's sequential scan keeps (e from 18 down, f from e down,
// replacing only on a strictly lower estimate: among equal estimates the
// first one scanned, i.e. the highest e, then the highest f).  Returns the
// class (e * (e + 1) / 2 + f), or kClassRD when the best estimate reaches
// the ALP-RD limit 48 * 32; without any pair that round-trips at least two
// samples the result is pair (0, 0) at the initial estimate, as the scan's.
__device__ int plain_search(const double *smp, int t, int *est_out, int *pair_out = nullptr) {
  constexpr int P = 2;  // pairs per round; three rounds cover ceil(190 / 32) = 6
  uint32_t key = 0xFFFFFFFFu;
#pragma unroll 1
  for (int round = 0; round < 3; ++round) {
    // per pair: 10^e, 10^-f, 10^f (as a double) and 10^-e in registers
    // (lanes index the constant tables differently, so they are read once)
    double m10e[P], mfrf[P], factd[P], frce[P], dmn[P], dmx[P];
    int64_t mn[P], mx[P];
    int cnt[P], pe[P], pf[P];
#pragma unroll
    for (int i = 0; i < P; ++i) {
      const int c = t + 32 * (round * P + i);
      const int e = c < kClassRD ? class_exp(c) : 0, f = c < kClassRD ? c - e * (e + 1) / 2 : 0;
      pe[i] = e;
      pf[i] = f;
      m10e[i] = c_f64_exp10[e];
      mfrf[i] = c_f64_frac[f];
      factd[i] = (double)c_f64_fact[f];
      frce[i] = c_f64_frac[e];
      dmn[i] = 1e300;
      dmx[i] = -1e300;
      mn[i] = INT64_MAX;
      mx[i] = INT64_MIN;
      cnt[i] = 0;
    }
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      const double x = smp[k];
#pragma unroll
      for (int i = 0; i < P; ++i) {
        const double tv = __dmul_rn(__dmul_rn(x, m10e[i]), mfrf[i]);
        const double r = __dsub_rn(__dadd_rn(tv, kMagic), kMagic);
        const double p = __dmul_rn(r, factd[i]);
        // |tv| < 2^51: r is the integer the reference's cast yields; |p| <
        // 2^53: the reference's integer product, converted, is p exactly;
        // -0.0 is the reference's "impossible" case
        if (fabs(tv) < 2251799813685248.0 && fabs(p) < 9007199254740992.0 &&
            __double_as_longlong(tv) != (long long)0x8000000000000000ull) {
          if (__dmul_rn(p, frce[i]) == x) {
            ++cnt[i];
            dmn[i] = fmin(dmn[i], r);
            dmx[i] = fmax(dmx[i], r);
          }
        } else {
          const int64_t q = impossible_f64(tv) ? (int64_t)kEncUpper : cvtt_s64(r);
          const double d = __dmul_rn(
              __ll2double_rn((long long)((uint64_t)q * (uint64_t)c_f64_fact[pf[i]])), frce[i]);
          if (d == x) {
            ++cnt[i];
            mn[i] = q < mn[i] ? q : mn[i];
            mx[i] = q > mx[i] ? q : mx[i];
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < P; ++i) {
      const int c = t + 32 * (round * P + i);
      if (c < kClassRD && cnt[i] >= 2) {
        int64_t lo = mn[i], hi = mx[i];
        if (dmn[i] <= dmx[i]) {
          const int64_t a = (int64_t)dmn[i], b = (int64_t)dmx[i];
          lo = a < lo ? a : lo;
          hi = b > hi ? b : hi;
        }
        const int est = 32 * count_bits64((uint64_t)hi - (uint64_t)lo) + (32 - cnt[i]) * 80;
        const uint32_t kk =
            ((uint32_t)est << 10) | ((uint32_t)(18 - pe[i]) << 5) | (uint32_t)(18 - pf[i]);
        key = kk < key ? kk : key;
      }
    }
  }
  key = __reduce_min_sync(0xffffffffu, key);
  int sbest = 32 * (64 + 16) + 32 * 64, fe = 0, ff = 0;
  if (key != 0xFFFFFFFFu) {
    sbest = (int)(key >> 10);
    fe = 18 - (int)((key >> 5) & 31);
    ff = 18 - (int)(key & 31);
  }
  if (est_out) *est_out = sbest;
  if (pair_out) *pair_out = pair_class(fe, ff);
  return sbest >= kRDLimitBits ? kClassRD : pair_class(fe, ff);
}

// Labels (the plain search's class) of every vector: one warp per vector.
__global__ void __launch_bounds__(256, 4) k_plain_labels(const double *__restrict__ vals,
                                                      size_t n_vecs, int16_t *labels,
                                                      int32_t *est) {
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  __shared__ double s_smp[8][32];
  double *smp = s_smp[threadIdx.x >> 5];
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    __syncwarp();
    smp[t] = vals[v * VEC + 32 * t];
    __syncwarp();
    int e;
    const int cls = plain_search(smp, t, &e);
    if (t == 0) {
      labels[v] = (int16_t)cls;
      if (est) est[v] = e;
    }
  }
}

// ---- vector encode ---------------------------------------------------------
// Thread t owns lane t % 16, values 32*(t/16) .. +31 of the lane (position
// lane + 16*(32*half + k)).  The encode runs in two kernels: the first
// analyses each vector under its chosen (e, f) (exceptions, the fill
// integer, base and width), the second, after the scan of the sizes,
// recomputes the integers and writes the packed words and exceptions
// straight to their final offsets.

// encode_simdized's exception test for one value: specials (inf, NaN,
// -0.0) are encoded as the upper bound and become exceptions.
__device__ __forceinline__ int64_t enc_checked(double x, double m10e, double mfrf, uint64_t fact,
                                               double frce, bool *is_exc) {
  const uint64_t bits = (uint64_t)__double_as_longlong(x);
  const bool special = ((bits & 0x7FFFFFFFFFFFFFFFull) >= 0x7FF0000000000000ull) ||
                       bits == 0x8000000000000000ull;
  const double a = special ? kEncUpper : x;
  const int64_t q = enc_stored(a, m10e, mfrf);
  *is_exc = dec_stored(q, fact, frce) != a;
  return q;
}

struct VecAnalysis {
  uint32_t mask;  // this thread's exceptions (bit k: value k of its 32)
  int n_exc;
  int bw;
  int64_t fill;   // the integer stored at exception positions
  uint64_t base;  // minimum of the stored integers
};

__device__ VecAnalysis analyze_vector(const double *__restrict__ vec, int e, int f, int t) {
  const int lane = t & 15, half = t >> 4;
  uint32_t exc_mask = 0;
  int first_ok = 1 << 30;
  int64_t mn = INT64_MAX, mx = INT64_MIN;
  const double m10e = c_f64_exp10[e], mfrf = c_f64_frac[f], frce = c_f64_frac[e];
  const uint64_t fact = (uint64_t)c_f64_fact[f];
  const double *src = vec + lane + 16 * 32 * half;
  // eight loads in flight at a time (each a whole 128-byte line per half
  // warp), few registers, so that many warps hide the latency
#pragma unroll 1
  for (int c = 0; c < 32; c += 8) {
    double xv[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) xv[i] = src[16 * (c + i)];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int k = c + i;
      const int p = lane + 16 * (32 * half + k);
      bool is_exc;
      const int64_t q = enc_checked(xv[i], m10e, mfrf, fact, frce, &is_exc);
      exc_mask |= (uint32_t)is_exc << k;
      if (!is_exc) {
        first_ok = min(first_ok, p);
        mn = q < mn ? q : mn;
        mx = q > mx ? q : mx;
      }
    }
  }
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) first_ok = min(first_ok, __shfl_xor_sync(0xffffffffu, first_ok, s));
  VecAnalysis a;
  a.mask = exc_mask;
  a.n_exc = __reduce_add_sync(0xffffffffu, __popc(exc_mask));
  // the first non-exception's integer (0 when every position, or every
  // position but the last, is an exception: encoder.hpp:361-367)
  a.fill = 0;
  if (first_ok < VEC && !(first_ok == VEC - 1 && a.n_exc == VEC - 1))
    a.fill = enc_value(vec[first_ok], f, e, false);
  if (exc_mask) {
    mn = a.fill < mn ? a.fill : mn;
    mx = a.fill > mx ? a.fill : mx;
  }
  mn = warp_min_s64(mn);
  mx = warp_max_s64(mx);
  a.bw = count_bits64((uint64_t)mx - (uint64_t)mn);
  a.base = (uint64_t)mn;
  return a;
}

// The bw 32-bit words of one thread: its 32 values (value k at position
// lane + 16 (32 half + k)), as offsets from the vector's base, are bits
// [32 half bw, 32 (half + 1) bw) of the lane's stream, so the words are the
// thread's alone.  Word m of lane l of the 64-bit stream lives at 32-bit
// index 2 l + 32 (m / 2) + m % 2, i.e. word w of this thread (m = half bw +
// w) at 16 m - 15 (m % 2): pa + 16 w for even w, pb + 16 w for odd w.  The
// values are loaded eight at a time (for each k the warp reads two whole
// 128-byte lines) and encoded with exceptions storing the fill integer;
// widths up to 32 take 32-bit shifts only.
__device__ __forceinline__ void pack_thread(const double *__restrict__ vec, uint32_t mask,
                                            int64_t fill, uint64_t base, double m10e,
                                            double mfrf, int bw, uint32_t *p32, int lane,
                                            int half) {
  const int oddm0 = half & bw & 1;
  uint32_t *pa = p32 + half * 16 * bw - (oddm0 ? 15 : 0);
  uint32_t *pb = p32 + half * 16 * bw - (oddm0 ? 0 : 15);
  const uint64_t vmask = bw >= 64 ? ~0ull : ((1ull << bw) - 1);
  const double *src = vec + lane + 16 * 32 * half;
  int w = 0;         // the next word
  uint32_t acc = 0;  // its pending low bits
  int nacc = 0;      // how many
  if (bw <= 32) {
#pragma unroll 1
    for (int c = 0; c < 32; c += 8) {
      double xv[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) xv[i] = src[16 * (c + i)];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k = c + i;
        const int64_t q = ((mask >> k) & 1u) ? fill : enc_stored(xv[i], m10e, mfrf);
        const uint32_t d = (uint32_t)(((uint64_t)q - base) & vmask);
        const uint32_t lo = acc | (d << nacc);
        nacc += bw;
        if (nacc >= 32) {
          ((w & 1) ? pb : pa)[16 * w] = lo;
          ++w;
          nacc -= 32;
          acc = nacc ? d >> (bw - nacc) : 0u;  // the bits of d past the word
        } else {
          acc = lo;
        }
      }
    }
  } else {
#pragma unroll 1
    for (int c = 0; c < 32; c += 8) {
      double xv[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) xv[i] = src[16 * (c + i)];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k = c + i;
        const int64_t q = ((mask >> k) & 1u) ? fill : enc_stored(xv[i], m10e, mfrf);
        const uint64_t d = ((uint64_t)q - base) & vmask;
        // (hi:lo) = acc | d << nacc holds nacc + bw (33..95) bits
        const uint64_t lo = (uint64_t)acc | (d << nacc);
        const uint32_t hi = nacc ? (uint32_t)(d >> (64 - nacc)) : 0u;
        int total = nacc + bw - 32;
        ((w & 1) ? pb : pa)[16 * w] = (uint32_t)lo;
        ++w;
        if (total >= 32) {
          ((w & 1) ? pb : pa)[16 * w] = (uint32_t)(lo >> 32);
          ++w;
          total -= 32;
          acc = hi;
        } else {
          acc = (uint32_t)(lo >> 32);
        }
        nacc = total;
      }
    }
  }
}

// Exceptions (value, position) of one vector in ascending position at `exc`
// / `pos`: positions of round r = 16 r + lane, rounds 0..31 come from half
// 0, rounds 32..63 from half 1; only rounds holding an exception are
// visited.  exc_mask is this thread's mask from the analysis.
__device__ __forceinline__ void write_exceptions(const double *__restrict__ vec, uint32_t exc_mask,
                                                 int t, double *exc, uint16_t *pos) {
  const int lane = t & 15, half = t >> 4;
  const uint32_t any0 = __reduce_or_sync(0xffffffffu, half == 0 ? exc_mask : 0u);
  const uint32_t any1 = __reduce_or_sync(0xffffffffu, half == 1 ? exc_mask : 0u);
  uint64_t rounds = (uint64_t)any0 | ((uint64_t)any1 << 32);
  int written = 0;
  while (rounds) {
    const int r = __ffsll((long long)rounds) - 1;
    rounds &= rounds - 1;
    const int h = r >> 5, k = r & 31;
    const bool mine = (half == h) && ((exc_mask >> k) & 1);
    const unsigned bal = __ballot_sync(0xffffffffu, mine);
    if (mine) {
      const int slot = written + __popc(bal & ((1u << t) - 1));
      const int p = lane + 16 * r;
      exc[slot] = vec[p];
      pos[slot] = (uint16_t)p;
    }
    written += __popc(bal);
  }
}

// Hybrid columns: vector v as ALP-RD, with a dictionary of its own built
// from its 32 samples (rd_encoder::init on the vector alone: the
// first-level sample of one vector is its values at stride 32), and its
// exceptions counted; its ALP entry is empty.
__device__ __forceinline__ void choose_rd(const double *__restrict__ vec, const double *smp,
                                          uint64_t *srt, size_t v, int t, EncodeSlots &sl,
                                          RDWork &rd) {
  rd_rank_sort<uint64_t>(reinterpret_cast<const uint64_t *>(smp), 32, srt, t);
  const RDChoice ch = rd_find_best<uint64_t, 32>(srt, 32, t);
  const RDLookup lk(ch);
  const int n_exc = rd_count_exceptions<uint64_t>(reinterpret_cast<const uint64_t *>(vec), lk, t);
  sl.exc_mask[v * 32 + t] = 0u;
  if (t < kRDDict) rd.dicts[v * kRDDict + t] = (uint16_t)(t < ch.dsize ? ch.entry : 0u);
  if (t == 0) {
    sl.bw[v] = 0;
    sl.base[v] = 0;
    sl.fill[v] = 0;
    sl.fac[v] = 0;
    sl.exp[v] = 0;
    sl.count[v] = 0;
    rd.scheme[v] = (uint8_t)FLSGPU_SCHEME_ALP_RD;
    rd.rbw[v] = (uint8_t)ch.rbw;
    rd.lbw[v] = (uint8_t)ch.lbw;
    rd.dsize[v] = (uint8_t)ch.dsize;
    rd.dict_idx[v] = (uint32_t)v;
    rd.count[v] = (uint16_t)n_exc;
    rd.sizes[v] = (uint32_t)(ch.rbw * 16);
    rd.sizes[rd.cap + v] = (uint32_t)(ch.lbw * 64);
    rd.sizes[2 * rd.cap + v] = (uint32_t)n_exc;
  }
}

// Hybrid columns: vector v is ALP; its ALP-RD entry is empty.
__device__ __forceinline__ void mark_alp(size_t v, int t, RDWork &rd) {
  if (t < kRDDict) rd.dicts[v * kRDDict + t] = 0;
  if (t == 0) {
    rd.scheme[v] = (uint8_t)FLSGPU_SCHEME_ALP;
    rd.rbw[v] = 0;
    rd.lbw[v] = 0;
    rd.dsize[v] = 0;
    rd.dict_idx[v] = (uint32_t)v;
    rd.count[v] = 0;
    rd.sizes[v] = 0;
    rd.sizes[rd.cap + v] = 0;
    rd.sizes[2 * rd.cap + v] = 0;
  }
}

// Parameters of every vector, one warp per vector.  mode 0: the plain
// search; mode 1: candidates (k per vector, network order) chosen among on
// the samples with the reference's second-level rule (encoder.hpp:237-300),
// and the plain search when no candidate is an ALP pair or the choice leaves
// more than `max_exc` exceptions in the vector.  Writes the vector's
// exponent, factor, width, base, exception count, fill integer and flags
// (bit 0: the plain search ran as fallback; bit 1: ALP-RD territory, or in
// a hybrid column: encoded as ALP-RD).
// HYBRID: the vectors that call for ALP-RD are encoded as ALP-RD (mode 0:
// the search's estimate reaches the ALP-RD limit, encoder.hpp:208-211;
// mode 1: the network's top class is ALP-RD and none of its proposed ALP
// pairs estimates below that limit on the samples).
template <bool HYBRID>
__global__ void __launch_bounds__(256, 4)
    k_alp_choose(const double *__restrict__ vals, size_t n_vecs, int mode,
                 const int16_t *__restrict__ cand, int k_cand, int max_exc, EncodeSlots sl,
                 RDWork rd) {
  __shared__ double s_smp[8][32];
  __shared__ uint64_t s_srt[HYBRID ? 8 : 1][32];
  double *smp = s_smp[threadIdx.x >> 5];
  uint64_t *srt = s_srt[HYBRID ? (threadIdx.x >> 5) : 0];
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const double *vec = vals + v * VEC;
    const double s = vec[32 * t];
    __syncwarp();
    smp[t] = s;
    __syncwarp();
    int cls = -1;
    bool fallback = false, rd_net = false;
    int best = 0;
    if (mode == 1) {
      int worse = 0, chosen = -1;
      for (int c = 0; c < k_cand; ++c) {
        const int pc = cand[v * k_cand + c];
        if (pc < 0 || pc >= kClassRD) continue;
        const int est = sample_estimate(s, class_exp(pc), class_fac(pc), false);
        if (chosen < 0) {
          best = est;
          chosen = pc;
          continue;
        }
        if (est >= best) {
          if (++worse == 2) break;
          continue;
        }
        best = est;
        chosen = pc;
        worse = 0;
      }
      cls = chosen;
      rd_net = cand[v * k_cand] == kClassRD;
      if (cls < 0) fallback = true;
    }
    if constexpr (HYBRID) {
      // the network calls for ALP-RD and no proposed ALP pair gets below
      // the limit on the samples
      if (mode == 1 && rd_net && (cls < 0 || best >= kRDLimitBits)) {
        choose_rd(vec, smp, srt, v, t, sl, rd);
        if (t == 0) sl.flags[v] = 2;
        continue;
      }
    }
    // A vector in ALP-RD territory is still encoded as ALP with the search's
    // best pair (most values become exceptions): the column stays an
    // ALPColumn, and the RD decision is reported through the flags.
    int pair = 0;
    if (mode == 0 || fallback) {
      cls = plain_search(smp, t, nullptr, &pair);
    } else {
      pair = cls;
    }
    if constexpr (HYBRID) {
      if (cls == kClassRD) {
        choose_rd(vec, smp, srt, v, t, sl, rd);
        if (t == 0) sl.flags[v] = (uint8_t)((fallback ? 1 : 0) | 2);
        continue;
      }
    }
    const bool rd_flag = HYBRID ? false : (cls == kClassRD || rd_net);
    int e = class_exp(pair), f = class_fac(pair);
    VecAnalysis a = analyze_vector(vec, e, f, t);
    // Fall back when the proposal leaves more than max_exc exceptions, ALP-RD
    // proposals included: their ALP pair is then the plain search's, so the
    // column's size never depends on how far the network's ALP candidates
    // are from the search's choice on high-exception vectors.
    // The search itself runs in k_alp_fallback over the listed vectors, so
    // that the warps of this kernel all carry the same load.
    if (mode == 1 && !fallback && a.n_exc > max_exc) {
      if (t == 0) {
        sl.fb_list[atomicAdd(sl.fb_count, 1u)] = (uint32_t)v;
        sl.flags[v] = (uint8_t)(1 | (rd_flag ? 2 : 0));
      }
      continue;
    }
    if constexpr (HYBRID) mark_alp(v, t, rd);
    sl.exc_mask[v * 32 + t] = a.mask;
    if (t == 0) {
      sl.bw[v] = (uint8_t)a.bw;
      sl.base[v] = a.base;
      sl.fill[v] = a.fill;
      sl.fac[v] = (uint8_t)f;
      sl.exp[v] = (uint8_t)e;
      sl.count[v] = (uint16_t)a.n_exc;
      sl.flags[v] = (uint8_t)((fallback ? 1 : 0) | (rd_flag ? 2 : 0));
    }
  }
}

// The plain search and analysis of the vectors k_alp_choose listed (their
// proposal left more than max_exc exceptions); one warp per listed vector.
// HYBRID: a vector the search sends to ALP-RD is encoded as ALP-RD.
template <bool HYBRID>
__global__ void __launch_bounds__(256, 4)
    k_alp_fallback(const double *__restrict__ vals, EncodeSlots sl, RDWork rd) {
  __shared__ double s_smp[8][32];
  __shared__ uint64_t s_srt[HYBRID ? 8 : 1][32];
  double *smp = s_smp[threadIdx.x >> 5];
  uint64_t *srt = s_srt[HYBRID ? (threadIdx.x >> 5) : 0];
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const size_t n = *sl.fb_count;
  for (size_t i = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const size_t v = sl.fb_list[i];
    const double *vec = vals + v * VEC;
    __syncwarp();
    smp[t] = vec[32 * t];
    __syncwarp();
    int pair;
    const int cls = plain_search(smp, t, nullptr, &pair);
    if constexpr (HYBRID) {
      if (cls == kClassRD) {
        choose_rd(vec, smp, srt, v, t, sl, rd);
        if (t == 0) sl.flags[v] = 3;
        continue;
      }
      mark_alp(v, t, rd);
    }
    const int e = class_exp(pair), f = class_fac(pair);
    const VecAnalysis a = analyze_vector(vec, e, f, t);
    sl.exc_mask[v * 32 + t] = a.mask;
    if (t == 0) {
      sl.bw[v] = (uint8_t)a.bw;
      sl.base[v] = a.base;
      sl.fill[v] = a.fill;
      sl.fac[v] = (uint8_t)f;
      sl.exp[v] = (uint8_t)e;
      sl.count[v] = (uint16_t)a.n_exc;
      if (HYBRID) sl.flags[v] = 1;
    }
  }
}

// Column statistics for the caller: totals[2] += fallbacks, totals[3] +=
// ALP-RD vectors, totals[4] += the sum of the bit widths.
__global__ void __launch_bounds__(256) k_encode_stats(const uint8_t *flags, const uint8_t *bw,
                                                      size_t n, size_t *totals) {
  size_t fb = 0, rd = 0, sbw = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    fb += flags[i] & 1;
    rd += (flags[i] >> 1) & 1;
    sbw += bw[i];
  }
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    fb += __shfl_xor_sync(0xffffffffu, fb, s);
    rd += __shfl_xor_sync(0xffffffffu, rd, s);
    sbw += __shfl_xor_sync(0xffffffffu, sbw, s);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd((unsigned long long *)&totals[2], (unsigned long long)fb);
    atomicAdd((unsigned long long *)&totals[3], (unsigned long long)rd);
    atomicAdd((unsigned long long *)&totals[4], (unsigned long long)sbw);
  }
}

// Exclusive scan of the per-vector sizes (packed words = bw * 16,
// exceptions) in three steps: per block of 1024 vectors (k_scan_local:
// offsets within the block, block totals), over the block totals
// (k_scan_blocks: one block; also the column totals), and the block offset
// added by k_alp_pack, which writes the final offsets.
__device__ __forceinline__ void block_excl_scan2(size_t &a, size_t &b, size_t *sa, size_t *sb,
                                                 size_t &tot_a, size_t &tot_b) {
  const int t = threadIdx.x & 31, w = threadIdx.x >> 5;
  size_t ia = a, ib = b;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const size_t ya = __shfl_up_sync(0xffffffffu, ia, o), yb = __shfl_up_sync(0xffffffffu, ib, o);
    if (t >= o) {
      ia += ya;
      ib += yb;
    }
  }
  if (t == 31) {
    sa[w] = ia;
    sb[w] = ib;
  }
  __syncthreads();
  if (w == 0) {
    size_t xa = t < (int)(blockDim.x >> 5) ? sa[t] : 0, xb = t < (int)(blockDim.x >> 5) ? sb[t] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const size_t ya = __shfl_up_sync(0xffffffffu, xa, o), yb = __shfl_up_sync(0xffffffffu, xb, o);
      if (t >= o) {
        xa += ya;
        xb += yb;
      }
    }
    sa[t] = xa;  // inclusive over warps
    sb[t] = xb;
  }
  __syncthreads();
  const size_t wa = w ? sa[w - 1] : 0, wb = w ? sb[w - 1] : 0;
  tot_a = sa[(blockDim.x >> 5) - 1];
  tot_b = sb[(blockDim.x >> 5) - 1];
  a = wa + ia - a;
  b = wb + ib - b;
}

__global__ void __launch_bounds__(1024) k_scan_local(const uint8_t *bw, const uint16_t *count,
                                                     size_t n, size_t *off_words, size_t *off_exc,
                                                     size_t *blk_words, size_t *blk_exc) {
  __shared__ size_t sa[32], sb[32];
  const size_t v = (size_t)blockIdx.x * 1024 + threadIdx.x;
  size_t a = v < n ? (size_t)bw[v] * 16 : 0, b = v < n ? count[v] : 0;
  size_t ta, tb;
  block_excl_scan2(a, b, sa, sb, ta, tb);
  if (v < n) {
    off_words[v] = a;
    off_exc[v] = b;
  }
  if (threadIdx.x == 0) {
    blk_words[blockIdx.x] = ta;
    blk_exc[blockIdx.x] = tb;
  }
}

__global__ void __launch_bounds__(1024) k_scan_blocks(size_t nb, size_t *blk_words,
                                                      size_t *blk_exc, size_t *totals) {
  __shared__ size_t sa[32], sb[32];
  size_t carry_a = 0, carry_b = 0;
  for (size_t base = 0; base < nb; base += 1024) {
    const size_t i = base + threadIdx.x;
    size_t a = i < nb ? blk_words[i] : 0, b = i < nb ? blk_exc[i] : 0;
    size_t ta, tb;
    block_excl_scan2(a, b, sa, sb, ta, tb);
    if (i < nb) {
      blk_words[i] = carry_a + a;
      blk_exc[i] = carry_b + b;
    }
    carry_a += ta;
    carry_b += tb;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    totals[0] = carry_a;
    totals[1] = carry_b;
  }
}


// Packing at the final offsets: one warp per vector; thread t loads its 32
// values straight from the column and writes its words of the lane stream.
// HYBRID: ALP-RD vectors write their right parts, dictionary indices and
// exceptions instead (rd_write_vector), and both sub-columns' offsets are
// made final for every vector.
template <bool HYBRID>
__global__ void __launch_bounds__(256, 4) k_alp_pack(const double *__restrict__ vals, size_t n_vecs,
                                                  EncodeSlots sl, size_t *off_words,
                                                  size_t *off_exc, const size_t *blk_words,
                                                  const size_t *blk_exc, uint64_t *packed,
                                                  double *exc, uint16_t *pos, RDWork rd) {
  const int t = threadIdx.x & 31, lane = t & 15, half = t >> 4;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const size_t nb = (rd.cap + 1023) / 1024;  // stride of the ALP-RD block offsets
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const double *vec = vals + v * VEC;
    const size_t ow = off_words[v] + blk_words[v >> 10], oe = off_exc[v] + blk_exc[v >> 10];
    if constexpr (HYBRID) {
      const size_t orr = rd.offs[v] + rd.blk[v >> 10];
      const size_t ol = rd.offs[rd.cap + v] + rd.blk[nb + (v >> 10)];
      const size_t oer = rd.offs[2 * rd.cap + v] + rd.blk[2 * nb + (v >> 10)];
      if (rd.scheme[v] == FLSGPU_SCHEME_ALP_RD) {
        const RDLookup lk(rd.dicts + v * kRDDict, rd.dsize[v], rd.rbw[v]);
        rd_write_vector<uint64_t>(reinterpret_cast<const uint64_t *>(vec), lk, rd.lbw[v], t,
                                  rd.right + orr, rd.left + ol, rd.exc + oer, rd.pos + oer);
      }
      __syncwarp();
      if (t == 0) {
        rd.offs[v] = orr;
        rd.offs[rd.cap + v] = ol;
        rd.offs[2 * rd.cap + v] = oer;
      }
    }
    const int bw = sl.bw[v];
    const double m10e = c_f64_exp10[sl.exp[v]], mfrf = c_f64_frac[sl.fac[v]];
    const int64_t fill = sl.fill[v];
    const uint64_t base = sl.base[v];
    const uint32_t mask = sl.exc_mask[v * 32 + t];
    if (t == 0) {
      off_words[v] = ow;  // the column's final offsets
      off_exc[v] = oe;
    }
    if (bw > 0)
      pack_thread(vec, mask, fill, base, m10e, mfrf, bw,
                  reinterpret_cast<uint32_t *>(packed + ow) + 2 * lane, lane, half);
    write_exceptions(vec, mask, t, exc + oe, pos + oe);
  }
}

static int warps_grid(size_t n_vecs) {
  return (int)persistent_blocks(n_vecs ? n_vecs : 1, 8, 4);
}

flsgpu_status run_plain_labels(const double *vals, size_t n_vecs, int16_t *labels, int32_t *est,
                               cudaStream_t s) {
  if (!n_vecs) return FLSGPU_OK;
  k_plain_labels<<<warps_grid(n_vecs), 256, 0, s>>>(vals, n_vecs, labels, est);
  note_launch();
  return check_cuda(cudaGetLastError(), "k_plain_labels");
}

flsgpu_status run_alp_encode(const double *vals, size_t n_vecs, int mode, const int16_t *cand,
                             int k_cand, int max_exc, const EncodeSlots &sl, size_t *off_words,
                             size_t *off_exc, size_t *totals, uint64_t *packed, double *exc,
                             uint16_t *pos, cudaStream_t s, RDWork *rd) {
  if (!n_vecs) return FLSGPU_OK;
  const bool hybrid = rd != nullptr;
  const RDWork rw = hybrid ? *rd : RDWork{};
  if (mode == 1) {
    flsgpu_status st = check_cuda(cudaMemsetAsync(sl.fb_count, 0, sizeof(uint32_t), s), "memset");
    if (st) return st;
  }
  if (hybrid)
    k_alp_choose<true><<<warps_grid(n_vecs), 256, 0, s>>>(vals, n_vecs, mode, cand, k_cand,
                                                          max_exc, sl, rw);
  else
    k_alp_choose<false><<<warps_grid(n_vecs), 256, 0, s>>>(vals, n_vecs, mode, cand, k_cand,
                                                           max_exc, sl, rw);
  if (mode == 1) {
    if (hybrid)
      k_alp_fallback<true><<<warps_grid(n_vecs), 256, 0, s>>>(vals, sl, rw);
    else
      k_alp_fallback<false><<<warps_grid(n_vecs), 256, 0, s>>>(vals, sl, rw);
    note_launch();
  }
  const size_t nb = (n_vecs + 1023) / 1024;
  k_scan_local<<<(unsigned)nb, 1024, 0, s>>>(sl.bw, sl.count, n_vecs, off_words, off_exc,
                                             sl.blk_words, sl.blk_exc);
  k_scan_blocks<<<1, 1024, 0, s>>>(nb, sl.blk_words, sl.blk_exc, totals);
  note_launch();
  if (hybrid) {
    // the ALP-RD sub-column's right words, left words and exceptions
    const size_t bstride = (rw.cap + 1023) / 1024;
    k_scan_n_local<3><<<(unsigned)nb, 1024, 0, s>>>(rw.sizes, rw.cap, n_vecs, rw.offs, rw.blk,
                                                    bstride);
    k_scan_n_blocks<3><<<1, 1024, 0, s>>>(nb, rw.blk, bstride, rw.totals);
    note_launch(2);
  }
  {
    flsgpu_status st = check_cuda(cudaMemsetAsync(totals + 2, 0, 3 * sizeof(size_t), s), "memset");
    if (st) return st;
  }
  k_encode_stats<<<persistent_blocks(n_vecs / 32 + 1, 8, 2), 256, 0, s>>>(sl.flags, sl.bw, n_vecs,
                                                                           totals);
  note_launch();
  if (hybrid)
    k_alp_pack<true><<<warps_grid(n_vecs), 256, 0, s>>>(
        vals, n_vecs, sl, off_words, off_exc, sl.blk_words, sl.blk_exc, packed, exc, pos, rw);
  else
    k_alp_pack<false><<<warps_grid(n_vecs), 256, 0, s>>>(
        vals, n_vecs, sl, off_words, off_exc, sl.blk_words, sl.blk_exc, packed, exc, pos, rw);
  note_launch(3);
  return check_cuda(cudaGetLastError(), "alp encode");
}

}  // namespace flsb200
