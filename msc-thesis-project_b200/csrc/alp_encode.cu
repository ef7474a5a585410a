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

namespace flsb200 {

static __constant__ double c_f64_exp10[19] = {1.0,  10.0, 100.0, 1e3,  1e4,  1e5,  1e6,
                                              1e7,  1e8,  1e9,   1e10, 1e11, 1e12, 1e13,
                                              1e14, 1e15, 1e16,  1e17, 1e18};

constexpr double kEncUpper = 9223372036854774784.0;  // constants.hpp:18
constexpr double kEncLower = -9223372036854774784.0;
constexpr double kMagic = 6755399441055744.0;         // 0x0018000000000000

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

// Exhaustive search over the 190 pairs (0 <= f <= e <= 18), tie rules of
// find_top_k_combinations; returns the class (pair index e*(e+1)/2 + f, or
// kClassRD when the best estimate reaches the ALP-RD limit 48*32).
__device__ int plain_search(double s, int *est_out, int *pair_out = nullptr) {
  int sbest = 32 * (64 + 16) + 32 * 64;
  int fe = 0, ff = 0;
  for (int e = 18; e >= 0; --e) {
    for (int f = e; f >= 0; --f) {
      const int est = sample_estimate(s, e, f, true);
      if (est < 0) continue;
      if (est < sbest || (est == sbest && fe < e) || (est == sbest && fe == e && ff < f)) {
        sbest = est;
        fe = e;
        ff = f;
      }
    }
  }
  if (est_out) *est_out = sbest;
  if (pair_out) *pair_out = pair_class(fe, ff);
  return sbest >= 48 * 32 ? kClassRD : pair_class(fe, ff);
}

// Labels (the plain search's class) of every vector: one warp per vector.
__global__ void __launch_bounds__(256) k_plain_labels(const double *__restrict__ vals,
                                                      size_t n_vecs, int16_t *labels,
                                                      int32_t *est) {
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const double s = vals[v * VEC + 32 * t];
    int e;
    const int cls = plain_search(s, &e);
    if (t == 0) {
      labels[v] = (int16_t)cls;
      if (est) est[v] = e;
    }
  }
}

// ---- vector encode ---------------------------------------------------------
// Thread t owns lane t % 16, values 32*(t/16) .. +31 of the lane (position
// lane + 16*(32*half + k)).  Returns the exception count; fills the packed
// FastLanes words (bw * 16 u64 at `packed`), the exceptions (value,
// position) in ascending position order at `exc`/`pos`, base and width.
__device__ int encode_vector(const double *__restrict__ vec, int e, int f, int t,
                             uint64_t *packed, double *exc, uint16_t *pos, uint64_t *base_out,
                             int *bw_out) {
  const int lane = t & 15, half = t >> 4;
  // pass 1: exceptions, first non-exception position, min / max of the
  // integers of the non-exceptions (the integers are recomputed in pass 2
  // rather than held: 32 int64 per thread would cap occupancy)
  uint32_t exc_mask = 0;
  int first_ok = 1 << 30;
  int64_t mn = INT64_MAX, mx = INT64_MIN;
#pragma unroll 4
  for (int k = 0; k < 32; ++k) {
    const int p = lane + 16 * (32 * half + k);
    const double x = vec[p];
    const uint64_t bits = (uint64_t)__double_as_longlong(x);
    const bool special = ((bits & 0x7FFFFFFFFFFFFFFFull) >= 0x7FF0000000000000ull) ||
                         bits == 0x8000000000000000ull;
    const double a = special ? kEncUpper : x;
    const int64_t q = enc_value(a, f, e, false);
    const bool is_exc = dec_value(q, f, e) != a;
    exc_mask |= (uint32_t)is_exc << k;
    if (!is_exc) {
      first_ok = min(first_ok, p);
      mn = q < mn ? q : mn;
      mx = q > mx ? q : mx;
    }
  }
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) first_ok = min(first_ok, __shfl_xor_sync(0xffffffffu, first_ok, s));
  const int n_exc = __reduce_add_sync(0xffffffffu, __popc(exc_mask));
  // the integer stored at exception positions: that of the first
  // non-exception (0 when every position, or every position but the last,
  // is an exception)
  int64_t fill = 0;
  if (first_ok < VEC && !(first_ok == VEC - 1 && n_exc == VEC - 1))
    fill = enc_value(vec[first_ok], f, e, false);
  if (exc_mask) {
    mn = fill < mn ? fill : mn;
    mx = fill > mx ? fill : mx;
  }
  mn = warp_min_s64(mn);
  mx = warp_max_s64(mx);
  const int bw = count_bits64((uint64_t)mx - (uint64_t)mn);
  const uint64_t base = (uint64_t)mn;
  // pass 2, pack: this thread's 32 values are bits [32*half*bw,
  // 32*(half+1)*bw) of the lane stream = its bw 32-bit words, owned by it
  // alone
  if (bw > 0) {
    uint32_t *p32 = reinterpret_cast<uint32_t *>(packed) + 2 * lane;
    const uint64_t mask = bw >= 64 ? ~0ull : ((1ull << bw) - 1);
    uint32_t acc = 0;  // pending low bits (< 32 of them)
    int nacc = 0, m = half * bw;
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      int64_t q = fill;
      if (!((exc_mask >> k) & 1)) {
        const double x = vec[lane + 16 * (32 * half + k)];
        q = enc_value(x, f, e, false);
      }
      const uint64_t d = ((uint64_t)q - base) & mask;
      // (hi:lo) = acc | d << nacc, total = nacc + bw bits (at most 95)
      uint64_t lo = (uint64_t)acc | (d << nacc);
      uint32_t hi = nacc ? (uint32_t)(d >> (64 - nacc)) : 0u;
      int total = nacc + bw;
      while (total >= 32) {
        p32[(m >> 1) * 32 + (m & 1)] = (uint32_t)lo;
        ++m;
        lo = (lo >> 32) | ((uint64_t)hi << 32);
        hi = 0;
        total -= 32;
      }
      acc = (uint32_t)lo;
      nacc = total;
    }
  }
  // exceptions in ascending position: positions of round r = 16 * r + lane,
  // rounds 0..31 come from half 0, rounds 32..63 from half 1; only rounds
  // holding an exception are visited
  int written = 0;
  if (n_exc) {
    const uint32_t any0 = __reduce_or_sync(0xffffffffu, half == 0 ? exc_mask : 0u);
    const uint32_t any1 = __reduce_or_sync(0xffffffffu, half == 1 ? exc_mask : 0u);
    uint64_t rounds = (uint64_t)any0 | ((uint64_t)any1 << 32);
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
  if (base_out) *base_out = base;
  if (bw_out) *bw_out = bw;
  return n_exc;
}

// One warp per vector.  mode 0: parameters from the plain search; mode 1:
// candidates (k per vector, network order) verified on the samples with the
// reference's second-level choice, plain search when the network proposes
// ALP-RD or the encode leaves more than `max_exc` exceptions.
__global__ void __launch_bounds__(256)
    k_alp_encode(const double *__restrict__ vals, size_t n_vecs, int mode,
                 const int16_t *__restrict__ cand, int k_cand, int max_exc, EncodeSlots sl) {
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const double *vec = vals + v * VEC;
    const double s = vec[32 * t];
    int cls = -1;
    bool fallback = false, rd_net = false;
    if (mode == 1) {
      // second-level choice among the proposed pairs (encoder.hpp:237-300)
      int best = 0, worse = 0, chosen = -1;
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
    // A vector in ALP-RD territory is still encoded as ALP with the search's
    // best pair (most values become exceptions): the column stays an
    // ALPColumn, and the RD decision is reported through the flags.
    int pair = 0;
    if (mode == 0 || fallback) {
      cls = plain_search(s, nullptr, &pair);
    } else {
      pair = cls;
    }
    const bool rd = cls == kClassRD || rd_net;
    int e = class_exp(pair), f = class_fac(pair);
    uint64_t base;
    int bw;
    int n_exc = encode_vector(vec, e, f, t, sl.packed + v * VEC, sl.exc + v * VEC,
                              sl.pos + v * VEC, &base, &bw);
    // Fall back when the proposal leaves more than max_exc exceptions, ALP-RD
    // proposals included: their ALP pair is then the plain search's, so the
    // column's size never depends on how far the network's ALP candidates
    // are from the search's choice on high-exception vectors.
    if (mode == 1 && !fallback && n_exc > max_exc) {
      // the proposal leaves too many exceptions: plain search and re-encode
      __syncwarp();
      fallback = true;
      int pc;
      plain_search(s, nullptr, &pc);
      e = class_exp(pc);
      f = class_fac(pc);
      n_exc = encode_vector(vec, e, f, t, sl.packed + v * VEC, sl.exc + v * VEC, sl.pos + v * VEC,
                            &base, &bw);
    }
    if (t == 0) {
      sl.bw[v] = (uint8_t)bw;
      sl.base[v] = base;
      sl.fac[v] = (uint8_t)f;
      sl.exp[v] = (uint8_t)e;
      sl.count[v] = (uint16_t)n_exc;
      sl.flags[v] = (uint8_t)((fallback ? 1 : 0) | (rd ? 2 : 0));
    }
  }
}

// Exclusive scan of per-vector sizes (packed words = bw * 16, exceptions)
// in one block; n_vecs up to a few million.
__global__ void __launch_bounds__(1024) k_scan_sizes(const uint8_t *bw, const uint16_t *count,
                                                     size_t n, size_t *off_words,
                                                     size_t *off_exc, size_t *totals) {
  __shared__ size_t s_w[1024], s_e[1024];
  const int tid = threadIdx.x;
  const size_t per = (n + 1023) / 1024;
  const size_t lo = tid * per, hi = min(n, lo + per);
  size_t sw = 0, se = 0;
  for (size_t i = lo; i < hi; ++i) {
    sw += (size_t)bw[i] * 16;
    se += count[i];
  }
  s_w[tid] = sw;
  s_e[tid] = se;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    size_t aw = 0, ae = 0;
    if (tid >= o) {
      aw = s_w[tid - o];
      ae = s_e[tid - o];
    }
    __syncthreads();
    s_w[tid] += aw;
    s_e[tid] += ae;
    __syncthreads();
  }
  size_t rw = s_w[tid] - sw, re = s_e[tid] - se;
  for (size_t i = lo; i < hi; ++i) {
    off_words[i] = rw;
    off_exc[i] = re;
    rw += (size_t)bw[i] * 16;
    re += count[i];
  }
  if (tid == 1023) {
    totals[0] = s_w[1023];
    totals[1] = s_e[1023];
  }
}

// Compaction into the contiguous column arrays: one warp per vector.
__global__ void __launch_bounds__(256) k_compact(EncodeSlots sl, size_t n_vecs,
                                                 const size_t *off_words, const size_t *off_exc,
                                                 uint64_t *packed, double *exc, uint16_t *pos) {
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const int nwd = sl.bw[v] * 16;
    const uint64_t *src = sl.packed + v * VEC;
    uint64_t *dst = packed + off_words[v];
    for (int i = t; i < nwd; i += 32) dst[i] = src[i];
    const int c = sl.count[v];
    for (int i = t; i < c; i += 32) {
      exc[off_exc[v] + i] = sl.exc[v * VEC + i];
      pos[off_exc[v] + i] = sl.pos[v * VEC + i];
    }
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
                             uint16_t *pos, cudaStream_t s) {
  if (!n_vecs) return FLSGPU_OK;
  k_alp_encode<<<warps_grid(n_vecs), 256, 0, s>>>(vals, n_vecs, mode, cand, k_cand, max_exc, sl);
  k_scan_sizes<<<1, 1024, 0, s>>>(sl.bw, sl.count, n_vecs, off_words, off_exc, totals);
  k_compact<<<warps_grid(n_vecs), 256, 0, s>>>(sl, n_vecs, off_words, off_exc, packed, exc, pos);
  note_launch(3);
  return check_cuda(cudaGetLastError(), "alp encode");
}

}  // namespace flsb200
