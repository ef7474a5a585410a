// unpack.cuh -- per-lane FastLanes bit unpacking, specialised per bit width.
//
// The reference decodes one value per call through runtime shifts and
// masks (BitUnpackerStatefulBranchless, src/flsgpu/fls.cuh:574-618).  Here
// every bit width is its own fully unrolled instantiation: all shift
// amounts and word indices are compile-time constants, a width switch is
// taken once per vector (uniform across the warp), and a thread decodes a
// whole lane (or half a lane for 64-bit types) from words it holds in
// registers.
#pragma once

#include "common.cuh"

namespace flsb200 {

// ---- 32-bit lanes: one thread per lane, 32 values -----------------------
// w[0..W-1] are the lane's packed words (line j at packed[j*32 + lane]).
template <int W, class F>
__device__ __forceinline__ void unpack_lane32(const uint32_t *w, F &&f) {
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    uint32_t v = 0;
    if (W > 0) {
      const int bit = k * W, j = bit >> 5, o = bit & 31;
      if (o + W <= 32)
        v = w[j] >> o;
      else
        v = funnel_r(w[j], w[j + 1], (uint32_t)o);
      v &= mask32<W>();
    }
    f(k, v);
  }
}

template <int W>
__device__ __forceinline__ void load_lane32(const uint32_t *vin, int lane, uint32_t *w) {
#pragma unroll
  for (int j = 0; j < W; ++j) w[j] = ld_stream_u32(vin + j * 32 + lane);
}

// ---- 64-bit lanes: two threads per lane ---------------------------------
// A 64-bit lane's bit stream, viewed as 32-bit words (low half of each
// 64-bit line first), holds values 0..31 in words [0, W) and values 32..63
// in words [W, 2W).  Thread t handles lane t % 16, half t / 16, so both
// halves decode with the same compile-time offsets.
template <int W>
__device__ __forceinline__ void load_half64(const uint64_t *vin, int lane, int half, uint32_t *w) {
  constexpr int L = W / 2 + 1;
  const int m0 = half * W;     // first 32-bit word of this half
  const int j0 = m0 >> 1;      // its 64-bit line
  const bool odd = (m0 & 1) != 0;
  uint64_t d[L];
#pragma unroll
  for (int i = 0; i < L; ++i) {
    const int j = j0 + i;
    d[i] = (j < W) ? ld_stream_u64(vin + j * 16 + lane) : 0ull;
  }
#pragma unroll
  for (int i = 0; i < W; ++i) {
    const uint32_t even_start = (i & 1) ? (uint32_t)(d[i >> 1] >> 32) : (uint32_t)d[i >> 1];
    const uint32_t odd_start =
        (i & 1) ? (uint32_t)d[(i + 1) >> 1] : (uint32_t)(d[i >> 1] >> 32);
    w[i] = odd ? odd_start : even_start;
  }
}

// Same stream words as load_half64, read as 32-bit words straight from
// global memory (the two halves of a 64-bit line are consecutive loads, so
// the second one hits L1): W live registers instead of ~2W.
template <int W>
__device__ __forceinline__ void load_half64_w32(const uint64_t *vin, int lane, int half,
                                                uint32_t *w) {
  const uint32_t *p = reinterpret_cast<const uint32_t *>(vin) + 2 * lane;
  const int m0 = half * W;
#pragma unroll
  for (int i = 0; i < W; ++i) {
    const int m = m0 + i;
    w[i] = __ldg(p + (m >> 1) * 32 + (m & 1));
  }
}

template <int W, class F>
__device__ __forceinline__ void unpack_half64(const uint32_t *w, F &&f) {
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    uint64_t v = 0;
    if (W > 0) {
      const int bit = k * W, j = bit >> 5, o = bit & 31;
      const int je = (bit + W - 1) >> 5;
      const uint32_t x0 = w[j];
      const uint32_t x1 = (je >= j + 1) ? w[j + 1] : 0u;
      const uint32_t x2 = (je >= j + 2) ? w[j + 2] : 0u;
      const uint32_t lo = o ? funnel_r(x0, x1, (uint32_t)o) : x0;
      uint32_t hi = 0;
      if (W > 32 - o) hi = o ? funnel_r(x1, x2, (uint32_t)o) : x1;
      v = (((uint64_t)hi << 32) | lo) & mask64<W>();
    }
    f(k, v);
  }
}

// Chunked form for wide values: the half-lane's 32 values are decoded as
// two runs of 16, each loading only the 64-bit lines it spans, with a
// compiler barrier between the runs so that at most ~W/2 + 2 packed words
// are live.  This lowers register pressure (and raises occupancy) at the
// price of exposing the second run's load latency to the warp.
template <int W, class F>
__device__ __forceinline__ void decode_half64_chunked(const uint64_t *vin, int lane, int half,
                                                      F &&f) {
  const int m0 = half * W;
  const bool odd = (m0 & 1) != 0;
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    // stream words [J0, J1] (relative to the half) hold values 16c .. 16c+15
    constexpr int CW = (W > 0) ? W : 1;
    const int J0 = (16 * c * W) >> 5;
    const int J1 = (16 * (c + 1) * W + 31) >> 5;  // one past the last word
    constexpr int NMAX = (16 * CW + 31) / 32 + 2;
    uint32_t w[NMAX];
    // 64-bit lines covering stream words m0+J0 .. m0+J1-1
    const int l0 = (m0 + J0) >> 1;
    uint64_t d[NMAX / 2 + 2];
#pragma unroll
    for (int i = 0; i < NMAX / 2 + 2; ++i) {
      const int j = l0 + i;
      const bool need = (2 * i) < (J1 - J0 + 2);
      d[i] = (need && j < W) ? ld_stream_u64(vin + j * 16 + lane) : 0ull;
    }
    // word J0 + i is 64-bit line l0 + ((s + i) >> 1), half (s + i) & 1,
    // where s = (m0 + J0) & 1 (odd iff half * W + J0 is odd)
    const bool s = (((J0 & 1) != 0) != odd);
#pragma unroll
    for (int i = 0; i < NMAX; ++i) {
      const uint32_t ev = (i & 1) ? (uint32_t)(d[i >> 1] >> 32) : (uint32_t)d[i >> 1];
      const uint32_t od = (i & 1) ? (uint32_t)d[(i + 1) >> 1] : (uint32_t)(d[i >> 1] >> 32);
      w[i] = s ? od : ev;
    }
#pragma unroll
    for (int k = 16 * c; k < 16 * c + 16; ++k) {
      uint64_t v = 0;
      if (W > 0) {
        const int bit = k * W, j = (bit >> 5) - J0, o = bit & 31;
        const int je = ((bit + W - 1) >> 5) - J0;
        const uint32_t x0 = w[j];
        const uint32_t x1 = (je >= j + 1) ? w[j + 1] : 0u;
        const uint32_t x2 = (je >= j + 2) ? w[j + 2] : 0u;
        const uint32_t lo = o ? funnel_r(x0, x1, (uint32_t)o) : x0;
        uint32_t hi = 0;
        if (W > 32 - o) hi = o ? funnel_r(x1, x2, (uint32_t)o) : x1;
        v = (((uint64_t)hi << 32) | lo) & mask64<W>();
      }
      f(k, v);
    }
    asm volatile("" ::: "memory");
  }
}

// ---- 16-bit lanes (ALP-RD left indices): one thread per lane pair -------
// 32-bit word j*32 + t holds 16-bit line j of lanes 2t (low) and 2t+1.
// Each 16-bit lane has 16 values; f(sub, k, v) receives lane 2t+sub.
template <int W>
__device__ __forceinline__ void load_pair16(const uint16_t *vin, int t, uint32_t *w) {
  const uint32_t *p = reinterpret_cast<const uint32_t *>(vin);
#pragma unroll
  for (int j = 0; j < W; ++j) w[j] = ld_stream_u32(p + j * 32 + t);
}

template <int W, class F>
__device__ __forceinline__ void unpack_pair16(const uint32_t *w, F &&f) {
#pragma unroll
  for (int sub = 0; sub < 2; ++sub) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      uint32_t v = 0;
      if (W > 0) {
        const int bit = k * W, j = bit >> 4, o = bit & 15;
        const uint32_t s0 = sub ? (w[j] >> 16) : (w[j] & 0xFFFFu);
        v = s0 >> o;
        if (o + W > 16) {
          const uint32_t s1 = sub ? (w[j + 1] >> 16) : (w[j + 1] & 0xFFFFu);
          v |= s1 << (16 - o);
        }
        v &= mask32<W>();
      }
      f(sub, k, v);
    }
  }
}

// ---- width dispatch ------------------------------------------------------
// Calls f(IntC<W>{}) for the runtime width w in [0, MAXW]; returns false
// when w is out of range.
template <int MAXW, int W = 0, class F>
__device__ __forceinline__ bool dispatch_width(int w, F &&f) {
  if constexpr (W > MAXW) {
    return false;
  } else {
    if (w == W) {
      f(IntC<W>{});
      return true;
    }
    return dispatch_width<MAXW, W + 1>(w, f);
  }
}

// Jump-table form of the same dispatch (one indirect branch).
#define FLSB_CASE(W)   \
  case W:              \
    f(IntC<W>{});      \
    return true;
#define FLSB_CASES_0_15                                                            \
  FLSB_CASE(0) FLSB_CASE(1) FLSB_CASE(2) FLSB_CASE(3) FLSB_CASE(4) FLSB_CASE(5)    \
  FLSB_CASE(6) FLSB_CASE(7) FLSB_CASE(8) FLSB_CASE(9) FLSB_CASE(10) FLSB_CASE(11)  \
  FLSB_CASE(12) FLSB_CASE(13) FLSB_CASE(14) FLSB_CASE(15)
#define FLSB_CASES_16_32                                                           \
  FLSB_CASE(16) FLSB_CASE(17) FLSB_CASE(18) FLSB_CASE(19) FLSB_CASE(20)            \
  FLSB_CASE(21) FLSB_CASE(22) FLSB_CASE(23) FLSB_CASE(24) FLSB_CASE(25)            \
  FLSB_CASE(26) FLSB_CASE(27) FLSB_CASE(28) FLSB_CASE(29) FLSB_CASE(30)            \
  FLSB_CASE(31) FLSB_CASE(32)
#define FLSB_CASES_33_64                                                           \
  FLSB_CASE(33) FLSB_CASE(34) FLSB_CASE(35) FLSB_CASE(36) FLSB_CASE(37)            \
  FLSB_CASE(38) FLSB_CASE(39) FLSB_CASE(40) FLSB_CASE(41) FLSB_CASE(42)            \
  FLSB_CASE(43) FLSB_CASE(44) FLSB_CASE(45) FLSB_CASE(46) FLSB_CASE(47)            \
  FLSB_CASE(48) FLSB_CASE(49) FLSB_CASE(50) FLSB_CASE(51) FLSB_CASE(52)            \
  FLSB_CASE(53) FLSB_CASE(54) FLSB_CASE(55) FLSB_CASE(56) FLSB_CASE(57)            \
  FLSB_CASE(58) FLSB_CASE(59) FLSB_CASE(60) FLSB_CASE(61) FLSB_CASE(62)            \
  FLSB_CASE(63) FLSB_CASE(64)

template <class F> __device__ __forceinline__ bool switch_width26(int w, F &&f) {
  switch (w) {
    FLSB_CASES_0_15
    FLSB_CASE(16) FLSB_CASE(17) FLSB_CASE(18) FLSB_CASE(19) FLSB_CASE(20) FLSB_CASE(21)
    FLSB_CASE(22) FLSB_CASE(23) FLSB_CASE(24) FLSB_CASE(25) FLSB_CASE(26)
    default: return false;
  }
}
template <class F> __device__ __forceinline__ bool switch_width16(int w, F &&f) {
  switch (w) { FLSB_CASES_0_15 FLSB_CASE(16) default: return false; }
}
template <class F> __device__ __forceinline__ bool switch_width32(int w, F &&f) {
  switch (w) { FLSB_CASES_0_15 FLSB_CASES_16_32 default: return false; }
}
template <class F> __device__ __forceinline__ bool switch_width64(int w, F &&f) {
  switch (w) { FLSB_CASES_0_15 FLSB_CASES_16_32 FLSB_CASES_33_64 default: return false; }
}

}  // namespace flsb200
