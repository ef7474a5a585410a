// alp_encode_f32.cu -- GPU ALP encoder for f32 columns (the float path of the
// reference's CPU encoder: encode_value / decode_value for float,
// src/alp/encoder.hpp:77-84, src/alp/decoder.hpp:124-127; the sampling search
// of find_top_k_combinations, encoder.hpp:134-230, over one vector's 32
// samples; encode_simdized, encoder.hpp:302-379; analyze_ffor,
// encoder.hpp:104-115; fls::ffor for u32).  Parameters are chosen per
// vector (the plain search); the column is an ALPColumn<float>.
//
// Per vector one warp, thread t = FastLanes lane t (values t + 32 k):
//   k_alp32_choose  the search: lane l evaluates the pairs l, l + 32, l + 64
//                   of the 66 (0 <= f <= e <= 10) on all 32 samples; one warp
//                   minimum over (estimate, 10 - e, 10 - f) keeps the pair the
//                   reference's scan keeps (strictly lower estimates replace,
//                   so among equals the first scanned: highest e, then f);
//                   then the analysis under that pair (exceptions, fill
//                   integer, base = signed minimum, width) and the sizes;
//   scan            packed words and exceptions, exclusive prefixes;
//   k_alp32_pack    each thread writes its lane's w stream words (FFOR
//                   against the base) and the exceptions in position order.
// Float arithmetic is separately rounded (__fmul_rn / __fadd_rn), and the
// float -> int32 conversion gives the x86 result of the reference's cast for
// out-of-range values (INT32_MIN), so the integers are the reference's.
#include "alp_learn.cuh"
#include "rd_encode.cuh"

namespace flsb200 {

static __constant__ float c_f32_exp10[11] = {1.0f,   10.0f,   100.0f,   1e3f,   1e4f,  1e5f,
                                             1e6f,   1e7f,    1e8f,     1e9f,   1e10f};

constexpr float kMagic32 = 12582912.0f;  // 2^23 + 2^22
constexpr double kEncUpper32 = 9223372036854774784.0;  // constants.hpp:18
constexpr int kPairs32 = 66;                           // 0 <= f <= e <= 10
constexpr int kExcBits32 = 32 + 16;                    // EXCEPTION_SIZE + position

__device__ __forceinline__ int32_t cvtt_s32(float x) {
  if (!(x >= -2147483648.0f && x < 2147483648.0f)) return INT32_MIN;
  return (int32_t)x;
}

__device__ __forceinline__ bool impossible_f32(float n) {
  return !isfinite(n) || (double)n > kEncUpper32 || (double)n < -kEncUpper32 ||
         (n == 0.0f && signbit(n));
}

// encode_value<float> (encoder.hpp:77-84): round(v * 10^e * 10^-f) by the
// magic-number add / subtract; safe: impossible inputs give the upper limit,
// whose cast to int32 is INT32_MIN.
__device__ __forceinline__ int32_t enc32(float v, int f, int e, bool safe) {
  const float t = __fmul_rn(__fmul_rn(v, c_f32_exp10[e]), c_f32_frac[f]);
  if (safe && impossible_f32(t)) return INT32_MIN;
  return cvtt_s32(__fsub_rn(__fadd_rn(t, kMagic32), kMagic32));
}
// decode_value<float> (decoder.hpp:124-127)
__device__ __forceinline__ float dec32(int32_t q, int f, int e) {
  return __fmul_rn(__int2float_rn((int32_t)((uint32_t)q * (uint32_t)c_f32_fact[f])),
                   c_f32_frac[e]);
}

__device__ __forceinline__ int count_bits32(uint32_t x) { return x ? 32 - __clz((int)x) : 0; }

// The per-vector search over the 32 samples smp[0..31]; returns the pair
// class e (e + 1) / 2 + f (the pair (0, 0) when no pair round-trips two
// samples, as the scan's initial choice); *rd: the best estimate reaches
// the ALP-RD limit (22 bits per value, RD_SIZE_THRESHOLD_LIMIT for float).
__device__ int plain_search32(const float *smp, int t, bool *rd) {
  uint32_t key = 0xFFFFFFFFu;
#pragma unroll 1
  for (int c = t; c < kPairs32; c += 32) {
    const int e = class_exp(c), f = c - e * (e + 1) / 2;
    int nonexc = 0;
    int32_t mn = INT32_MAX, mx = INT32_MIN;
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      const float a = smp[k];
      const int32_t q = enc32(a, f, e, true);
      if (dec32(q, f, e) == a) {
        ++nonexc;
        mn = q < mn ? q : mn;
        mx = q > mx ? q : mx;
      }
    }
    if (nonexc < 2) continue;
    const uint32_t est = 32u * (uint32_t)count_bits32((uint32_t)mx - (uint32_t)mn) +
                         (uint32_t)(32 - nonexc) * kExcBits32;
    const uint32_t k = (est << 8) | ((uint32_t)(10 - e) << 4) | (uint32_t)(10 - f);
    key = k < key ? k : key;
  }
  key = __reduce_min_sync(0xffffffffu, key);
  *rd = key == 0xFFFFFFFFu || (key >> 8) >= 22u * 32u;
  if (key == 0xFFFFFFFFu) return 0;
  const int e = 10 - (int)((key >> 4) & 15u), f = 10 - (int)(key & 15u);
  return pair_class(e, f);
}


__global__ void __launch_bounds__(256, 4) k_alp32_choose(const float *__restrict__ vals,
                                                         size_t n_vecs, Enc32Slots sl) {
  __shared__ float s_smp[8][32];
  float *smp = s_smp[threadIdx.x >> 5];
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const float *vec = vals + v * VEC;
    __syncwarp();
    smp[t] = vec[32 * t];
    __syncwarp();
    bool rd;
    const int cls = plain_search32(smp, t, &rd);
    if (rd && t == 0) atomicAdd(reinterpret_cast<unsigned long long *>(sl.n_rd), 1ull);
    const int e = class_exp(cls), f = cls - e * (e + 1) / 2;
    // encode_simdized: specials (inf, NaN, -0.0) are encoded as the upper
    // limit and become exceptions; an exception's integer is the fill
    uint32_t mask = 0;
    int first_ok = 1 << 30;
    int32_t mn = INT32_MAX, mx = INT32_MIN;
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      const float x = vec[t + 32 * k];
      const uint32_t b = __float_as_uint(x);
      const bool special = (b & 0x7FFFFFFFu) >= 0x7F800000u || b == 0x80000000u;
      const float a = special ? (float)kEncUpper32 : x;
      const int32_t q = enc32(a, f, e, false);
      if (dec32(q, f, e) != a) {
        mask |= 1u << k;
      } else {
        first_ok = min(first_ok, t + 32 * k);
        mn = q < mn ? q : mn;
        mx = q > mx ? q : mx;
      }
    }
    first_ok = __reduce_min_sync(0xffffffffu, first_ok);
    const int n_exc = __reduce_add_sync(0xffffffffu, __popc(mask));
    // the integer at the first non-exception position (0 when every
    // position, or every position but the last, is an exception:
    // encoder.hpp:361-367)
    int32_t fill = 0;
    if (first_ok < VEC && !(first_ok == VEC - 1 && n_exc == VEC - 1))
      fill = enc32(vec[first_ok], f, e, false);
    if (mask) {
      mn = fill < mn ? fill : mn;
      mx = fill > mx ? fill : mx;
    }
    mn = __reduce_min_sync(0xffffffffu, mn);
    mx = __reduce_max_sync(0xffffffffu, mx);
    const int bw = count_bits32((uint32_t)mx - (uint32_t)mn);
    sl.exc_mask[v * 32 + t] = mask;
    if (t == 0) {
      sl.bw[v] = (uint8_t)bw;
      sl.base[v] = (uint32_t)mn;
      sl.fill[v] = fill;
      sl.fac[v] = (uint8_t)f;
      sl.exp[v] = (uint8_t)e;
      sl.count[v] = (uint16_t)n_exc;
      sl.sizes[v] = (uint32_t)bw * 32u;
      sl.sizes[sl.stride + v] = (uint32_t)n_exc;
    }
  }
}

__global__ void __launch_bounds__(256, 4) k_alp32_pack(const float *__restrict__ vals,
                                                       size_t n_vecs, Enc32Slots sl, size_t *offs,
                                                       const size_t *blk, size_t bstride,
                                                       uint32_t *packed, float *exc,
                                                       uint16_t *pos) {
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const float *vec = vals + v * VEC;
    const size_t ow = offs[v] + blk[v >> 10];
    const size_t oe = offs[sl.stride + v] + blk[bstride + (v >> 10)];
    const int bw = sl.bw[v], e = sl.exp[v], f = sl.fac[v];
    const uint32_t base = sl.base[v];
    const int32_t fill = sl.fill[v];
    const uint32_t mask = sl.exc_mask[v * 32 + t];
    if (bw > 0) {
      uint64_t acc = 0;
      int fillb = 0, word = 0;
      const uint32_t vmask = bw >= 32 ? 0xFFFFFFFFu : ((1u << bw) - 1u);
#pragma unroll 4
      for (int k = 0; k < 32; ++k) {
        const int32_t q = ((mask >> k) & 1u) ? fill : enc32(vec[t + 32 * k], f, e, false);
        acc |= (uint64_t)(((uint32_t)q - base) & vmask) << fillb;
        fillb += bw;
        if (fillb >= 32) {
          packed[ow + (size_t)(word++) * 32 + t] = (uint32_t)acc;
          acc >>= 32;
          fillb -= 32;
        }
      }
    }
    // exceptions in position order: round k holds positions 32 k .. 32 k + 31
    int written = 0;
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      const bool mine = (mask >> k) & 1u;
      const unsigned bal = __ballot_sync(0xffffffffu, mine);
      if (mine) {
        const int slot = written + __popc(bal & ((1u << t) - 1u));
        exc[oe + slot] = vec[t + 32 * k];
        pos[oe + slot] = (uint16_t)(t + 32 * k);
      }
      written += __popc(bal);
    }
    __syncwarp();
    if (t == 0) {
      offs[v] = ow;
      offs[sl.stride + v] = oe;
    }
  }
}

// Launches the f32 encode; offs / blk / totals are the scan's arrays
// ([2][stride], [2][bstride], [2]).
flsgpu_status run_alp_encode_f32(const float *vals, size_t n_vecs, const Enc32Slots &sl,
                                 size_t *offs, size_t *blk, size_t bstride, size_t *totals,
                                 uint32_t *packed, float *exc, uint16_t *pos, cudaStream_t s) {
  if (!n_vecs) return FLSGPU_OK;
  const unsigned grid = persistent_blocks(n_vecs, 8, 4);
  k_alp32_choose<<<grid, 256, 0, s>>>(vals, n_vecs, sl);
  const size_t nb = (n_vecs + 1023) / 1024;
  k_scan_n_local<2><<<(unsigned)nb, 1024, 0, s>>>(sl.sizes, sl.stride, n_vecs, offs, blk, bstride);
  k_scan_n_blocks<2><<<1, 1024, 0, s>>>(nb, blk, bstride, totals);
  k_alp32_pack<<<grid, 256, 0, s>>>(vals, n_vecs, sl, offs, blk, bstride, packed, exc, pos);
  note_launch(4);
  return check_cuda(cudaGetLastError(), "f32 ALP encode");
}

}  // namespace flsb200
