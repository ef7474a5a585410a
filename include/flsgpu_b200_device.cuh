/*
 * flsgpu_b200_device.cuh -- device-side decoders for use inside user kernels.
 *
 * The reference lets a kernel decode a vector in registers through its
 * decompressor concept (src/flsgpu/structs.cuh:24-31):
 *     auto it = Decompressor(column, vector_index, lane);
 *     for (...) it.unpack_next_into(registers);
 * (FFORDecompressor / BPDecompressor, src/flsgpu/fls.cuh:620-650;
 * ALPDecompressor, src/flsgpu/alp.cuh:463-485), with one thread per
 * FastLanes lane (lane = threadIdx.x % N_LANES, src/engine/device-utils.cuh:
 * 77-99).  This header provides the same interface over the C ABI's column
 * descriptors (include/flsgpu_b200.h): each call of unpack_next_into writes
 * the lane's next UNPACK_N_VALUES values; value k of lane l is element
 * l + k * N_LANES of the vector.  Exceptions of ALP columns are patched into
 * the values as they are produced, so the registers hold the decoded column
 * (same bit patterns as flsgpu_decompress_*).
 *
 * Header-only; include from a .cu file compiled for sm_100a.  The decoders
 * are plain stateful readers (a word index and a bit offset per lane): they
 * serve kernels that consume values in registers; the library's own decode
 * kernels (flsgpu_decompress_*) are the fast path to memory.
 */
#ifndef FLSGPU_B200_DEVICE_CUH
#define FLSGPU_B200_DEVICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "flsgpu_b200.h"

namespace flsgpu_b200 {
namespace device {

template <typename T> struct lane_traits;
template <> struct lane_traits<uint32_t> { using U = uint32_t; static constexpr unsigned N_LANES = 32; };
template <> struct lane_traits<uint64_t> { using U = uint64_t; static constexpr unsigned N_LANES = 16; };
template <> struct lane_traits<float> { using U = uint32_t; static constexpr unsigned N_LANES = 32; };
template <> struct lane_traits<double> { using U = uint64_t; static constexpr unsigned N_LANES = 16; };

/* Values per lane: 32 for 32-bit types, 64 for 64-bit types. */
template <typename T> __host__ __device__ constexpr unsigned values_per_lane() {
  return 1024u / lane_traits<T>::N_LANES;
}

/* ALP tables (src/alp/constants.hpp): 10^e as doubles / floats for the
 * fraction index, 10^f as integers for the factor index. */
namespace detail {
__device__ __forceinline__ double f64_frac(int e) {
  const double t[21] = {1.0,   0.1,   0.01,  0.001, 0.0001, 1e-5,  1e-6,  1e-7,  1e-8,  1e-9, 1e-10,
                        1e-11, 1e-12, 1e-13, 1e-14, 1e-15,  1e-16, 1e-17, 1e-18, 1e-19, 1e-20};
  return t[e];
}
__device__ __forceinline__ float f32_frac(int e) {
  const float t[11] = {1.0f, 0.1f, 0.01f, 0.001f, 0.0001f, 1e-5f, 1e-6f, 1e-7f, 1e-8f, 1e-9f, 1e-10f};
  return t[e];
}
__device__ __forceinline__ uint64_t pow10_u64(int f) {
  uint64_t x = 1;
  for (int i = 0; i < f; ++i) x *= 10u;
  return x;
}
}  // namespace detail

/* One lane's FastLanes bit stream: value k occupies bits [k w, (k + 1) w),
 * least significant first; stream word j of lane l is packed[j * N_LANES + l]. */
template <typename U> struct LaneReader {
  static constexpr unsigned BITS = sizeof(U) * 8;
  const U *in;      /* the lane's word 0 */
  unsigned n_lanes;
  unsigned w, bit;
  U mask;
  __device__ __forceinline__ LaneReader(const U *vec_packed, unsigned lane, unsigned n_lanes_,
                                        unsigned width)
      : in(vec_packed + lane), n_lanes(n_lanes_), w(width), bit(0),
        mask(width >= BITS ? ~U(0) : (U)((U(1) << width) - 1)) {}
  __device__ __forceinline__ U next() {
    if (w == 0) return 0;
    const unsigned j = bit / BITS, o = bit % BITS;
    U v = in[(size_t)j * n_lanes] >> o;
    if (o + w > BITS) v |= in[(size_t)(j + 1) * n_lanes] << (BITS - o);
    bit += w;
    return v & mask;
  }
};

/* BPDecompressor (fls.cuh:620-633): T = uint32_t or uint64_t. */
template <typename T, unsigned UNPACK_N_VALUES = 1> struct BPDecompressor {
  using U = typename lane_traits<T>::U;
  LaneReader<U> r;
  __device__ __forceinline__ BPDecompressor(const flsgpu_bp_column &c, size_t vector_index,
                                            unsigned lane)
      : r(reinterpret_cast<const U *>(c.packed_array) + c.vector_offsets[vector_index], lane,
          lane_traits<T>::N_LANES, c.bit_widths[vector_index]) {}
  __device__ __forceinline__ void unpack_next_into(T *out) {
#pragma unroll
    for (unsigned i = 0; i < UNPACK_N_VALUES; ++i) out[i] = (T)r.next();
  }
};

/* FFORDecompressor (fls.cuh:635-650): value + the vector's base. */
template <typename T, unsigned UNPACK_N_VALUES = 1> struct FFORDecompressor {
  using U = typename lane_traits<T>::U;
  LaneReader<U> r;
  U base;
  __device__ __forceinline__ FFORDecompressor(const flsgpu_ffor_column &c, size_t vector_index,
                                              unsigned lane)
      : r(reinterpret_cast<const U *>(c.bp.packed_array) + c.bp.vector_offsets[vector_index],
          lane, lane_traits<T>::N_LANES, c.bp.bit_widths[vector_index]),
        base(reinterpret_cast<const U *>(c.bases)[vector_index]) {}
  __device__ __forceinline__ void unpack_next_into(T *out) {
#pragma unroll
    for (unsigned i = 0; i < UNPACK_N_VALUES; ++i) out[i] = (T)(U)(r.next() + base);
  }
};

namespace detail {
/* ALPFunctor (alp.cuh:40-45): (T)(INT_T)((u + base) * factor) * fraction,
 * unsigned wraparound, one round-to-nearest conversion and multiply. */
template <typename T> struct AlpTransform;
template <> struct AlpTransform<double> {
  uint64_t base, fact;
  double frac;
  __device__ __forceinline__ void init(const void *factors, const void *fractions, uint64_t b, int fi,
                                       int ei) {
    base = b;
    fact = factors ? (uint64_t)reinterpret_cast<const int64_t *>(factors)[fi] : pow10_u64(fi);
    frac = fractions ? reinterpret_cast<const double *>(fractions)[ei] : f64_frac(ei);
  }
  __device__ __forceinline__ double operator()(uint64_t u) const {
    return __dmul_rn(__ll2double_rn((long long)((u + base) * fact)), frac);
  }
};
template <> struct AlpTransform<float> {
  uint32_t base, fact;
  float frac;
  __device__ __forceinline__ void init(const void *factors, const void *fractions, uint32_t b, int fi,
                                       int ei) {
    base = b;
    fact = factors ? (uint32_t)reinterpret_cast<const int32_t *>(factors)[fi]
                   : (uint32_t)pow10_u64(fi);
    frac = fractions ? reinterpret_cast<const float *>(fractions)[ei] : f32_frac(ei);
  }
  __device__ __forceinline__ float operator()(uint32_t u) const {
    return __fmul_rn(__int2float_rn((int32_t)((u + base) * fact)), frac);
  }
};
}  // namespace detail

/* ALPDecompressor (alp.cuh:463-485) over an ALPColumn: T = float or double.
 * The vector's exceptions are sorted by position; a cursor walks them as
 * the lane's positions (lane + k * N_LANES) grow, so a lane reads the list
 * once per vector. */
template <typename T, unsigned UNPACK_N_VALUES = 1> struct ALPDecompressor {
  using U = typename lane_traits<T>::U;
  static constexpr unsigned N = lane_traits<T>::N_LANES;
  LaneReader<U> r;
  detail::AlpTransform<T> xf;
  const T *exc;
  const uint16_t *pos;
  unsigned n_exc, cur, lane, k;
  __device__ __forceinline__ ALPDecompressor(const flsgpu_alp_column &c, size_t vector_index,
                                             unsigned lane_)
      : r(reinterpret_cast<const U *>(c.ffor.bp.packed_array) +
              c.ffor.bp.vector_offsets[vector_index],
          lane_, N, c.ffor.bp.bit_widths[vector_index]),
        exc(reinterpret_cast<const T *>(c.exceptions) + c.exceptions_offsets[vector_index]),
        pos(c.positions + c.exceptions_offsets[vector_index]),
        n_exc(c.counts ? c.counts[vector_index] : 0u), cur(0), lane(lane_), k(0) {
    xf.init(c.factors, c.fractions, reinterpret_cast<const U *>(c.ffor.bases)[vector_index],
            c.factor_indices[vector_index], c.fraction_indices[vector_index]);
  }
  __device__ __forceinline__ void unpack_next_into(T *out) {
#pragma unroll
    for (unsigned i = 0; i < UNPACK_N_VALUES; ++i, ++k) {
      T v = xf(r.next());
      const unsigned p = lane + k * N;
      while (cur < n_exc && pos[cur] < p) ++cur;
      if (cur < n_exc && pos[cur] == p) v = exc[cur];
      out[i] = v;
    }
  }
};

/* The same over an ALPExtendedColumn: the lane's own exceptions are
 * offsets_counts[v * N_LANES + lane] = (count << 10) | offset into the
 * vector's list (the count taken as stored: 6 bits). */
template <typename T, unsigned UNPACK_N_VALUES = 1> struct ALPExtendedDecompressor {
  using U = typename lane_traits<T>::U;
  static constexpr unsigned N = lane_traits<T>::N_LANES;
  LaneReader<U> r;
  detail::AlpTransform<T> xf;
  const T *exc;
  const uint16_t *pos;
  unsigned n_exc, cur, lane, k;
  __device__ __forceinline__ ALPExtendedDecompressor(const flsgpu_alpx_column &c,
                                                     size_t vector_index, unsigned lane_)
      : r(reinterpret_cast<const U *>(c.ffor.bp.packed_array) +
              c.ffor.bp.vector_offsets[vector_index],
          lane_, N, c.ffor.bp.bit_widths[vector_index]),
        cur(0), lane(lane_), k(0) {
    const uint16_t oc = c.offsets_counts ? c.offsets_counts[vector_index * N + lane_] : 0;
    const size_t first = c.exceptions_offsets[vector_index] + (oc & 1023u);
    exc = reinterpret_cast<const T *>(c.exceptions) + first;
    pos = c.positions + first;
    n_exc = oc >> 10;
    xf.init(c.factors, c.fractions, reinterpret_cast<const U *>(c.ffor.bases)[vector_index],
            c.factor_indices[vector_index], c.fraction_indices[vector_index]);
  }
  __device__ __forceinline__ void unpack_next_into(T *out) {
#pragma unroll
    for (unsigned i = 0; i < UNPACK_N_VALUES; ++i, ++k) {
      T v = xf(r.next());
      const unsigned p = lane + k * N;
      while (cur < n_exc && pos[cur] < p) ++cur;
      if (cur < n_exc && pos[cur] == p) v = exc[cur];
      out[i] = v;
    }
  }
};

}  // namespace device
}  // namespace flsgpu_b200

#endif /* FLSGPU_B200_DEVICE_CUH */
