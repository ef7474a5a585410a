#pragma once
// kernels.cuh -- column kernels: full decompression, decode fused with a sum,
// magic-value scan, synthetic compute, multi-column scan.
//
// Work mapping: one warp decodes one 1024-value vector at a time and walks
// the column with a grid stride over a persistent grid (a whole number of
// waves on the SMs).  Thread t owns lane t (32-bit types) or half of lane
// t % 16 (64-bit types, values 32*(t/16) .. +31), so every warp-wide load of
// a packed line and every warp-wide store of a decoded row is a contiguous
// 128-byte segment.  The reference instead maps one thread to one lane and
// one value per call (src/engine/device-utils.cuh:77-120).
#include <algorithm>

#include "common.cuh"
#include "autotune_table.h"
#include "unpack.cuh"

namespace flsb200 {

enum Kind { K_BP = 0, K_FFOR = 1, K_ALP = 2, K_ALPX = 3 };
enum Sink { S_STORE = 0, S_SUM = 1, S_QUERY = 2, S_COMPUTE = 3, S_ALLEQ = 4 };

template <typename T> struct UintOf;
template <> struct UintOf<uint32_t> { using U = uint32_t; using I = int32_t; };
template <> struct UintOf<uint64_t> { using U = uint64_t; using I = int64_t; };
template <> struct UintOf<float> { using U = uint32_t; using I = int32_t; };
template <> struct UintOf<double> { using U = uint64_t; using I = int64_t; };

struct ColumnParams {
  size_t n_values, n_vecs;
  const void *packed;
  const uint8_t *bw;
  const size_t *offs;
  const void *bases;
  const void *factors, *fractions;
  const uint8_t *fac_idx, *exp_idx;
  const size_t *exc_offs;
  const void *exc;
  const uint16_t *pos;
  const uint16_t *counts;  // ALPColumn
  const uint16_t *oc;      // ALPExtendedColumn
  int patch;
  size_t n_packed;         // 0: unchecked
};

struct KernelParams {
  ColumnParams c;
  uint32_t *d_status;
  void *out;               // S_STORE
  uint64_t *sum_u64;       // S_SUM integers
  double *partials;        // S_SUM float: one per vector
  uint8_t *found;          // S_QUERY / S_COMPUTE / S_ALLEQ
  uint64_t magic;          // bit pattern of the query value
  uint32_t n_rep;          // S_COMPUTE
  uint64_t runtime_zero;   // S_COMPUTE
  uint64_t prefetch[2];    // bit w: L2-prefetch the next vector's packed lines when its width is w
};

// ---- value transforms (functors of the reference) ------------------------
// BPFunctor / FFORFunctor, src/flsgpu/fls.cuh:16-41.
template <typename U> struct XInt {
  U base;
  __device__ __forceinline__ U operator()(U u) const { return u + base; }
};
// ALPFunctor, src/flsgpu/alp.cuh:40-45: (T)(INT_T)((u + base) * factor) * frac
// with unsigned wraparound; conversion and multiply are single RN ops, so
// the result is the CPU falp's bit for bit.
struct XAlpF32 {
  uint32_t base, fact;
  float frac;
  __device__ __forceinline__ float operator()(uint32_t u) const {
    return __fmul_rn(__int2float_rn((int32_t)((u + base) * fact)), frac);
  }
};
struct XAlpF64 {
  uint64_t base, fact;
  double frac;
  __device__ __forceinline__ double operator()(uint64_t u) const {
    return __dmul_rn(__ll2double_rn((long long)((u + base) * fact)), frac);
  }
};

template <typename T, int KIND> struct XformOf { using type = XInt<typename UintOf<T>::U>; };
template <int KIND> struct XformOf<float, KIND> { using type = XAlpF32; };
template <int KIND> struct XformOf<double, KIND> { using type = XAlpF64; };

template <typename T> __device__ __forceinline__ T from_bits(uint64_t b) {
  if constexpr (sizeof(T) == 4) {
    const uint32_t x = (uint32_t)b;
    return *reinterpret_cast<const T *>(&x);
  } else {
    return *reinterpret_cast<const T *>(&b);
  }
}

__device__ __forceinline__ void flag_status(uint32_t *s, uint32_t f) {
  if (s) atomicOr(s, f);
}

// Per-vector metadata, loaded one vector ahead of its use (the loads of
// vector i + stride are in flight while vector i is decoded).
template <typename T> struct Meta {
  using U = typename UintOf<T>::U;
  size_t off;
  U base;
  int w;
  int fi, ei;
  uint32_t ecnt;  // ALPColumn: the vector's exception count (0 when not patched)
  size_t eo;      // ALPColumn: index of its first exception
};

template <typename T, int KIND>
__device__ __forceinline__ Meta<T> load_meta(const ColumnParams &c, size_t vi, int lane = -1) {
  using U = typename UintOf<T>::U;
  Meta<T> m;
  m.w = c.bw[vi];
  m.off = c.offs[vi];
  m.base = (KIND == K_BP) ? U(0) : reinterpret_cast<const U *>(c.bases)[vi];
  if constexpr (std::is_floating_point<T>::value) {
    m.fi = c.fac_idx[vi];
    m.ei = c.exp_idx[vi];
  } else {
    m.fi = m.ei = 0;
  }
  m.ecnt = 0;
  m.eo = 0;
  if constexpr (KIND == K_ALP) {
    if (c.patch && c.counts) {
      m.ecnt = c.counts[vi];
      m.eo = c.exc_offs[vi];
    }
  } else if constexpr (KIND == K_ALPX) {
    // ALPExtendedColumn, given the lane: that lane's (count << 10 | offset)
    // word (the vector's count is their u16 sum, taken at the patch)
    constexpr int NL = Lanes<typename UintOf<T>::U>::N;
    if (c.patch && c.oc && lane >= 0) {
      m.ecnt = lane < NL ? c.oc[vi * NL + lane] : 0u;
      m.eo = c.exc_offs[vi];
    }
  }
  return m;
}

// Validates metadata and builds the transform; false = skip the vector.
template <typename T, int KIND>
__device__ __forceinline__ bool setup_from_meta(const ColumnParams &c, uint32_t *d_status,
                                                const Meta<T> &m, int lane,
                                                const typename UintOf<T>::U *&vin, int &w,
                                                typename XformOf<T, KIND>::type &xf) {
  using U = typename UintOf<T>::U;
  constexpr int MAXW = sizeof(U) * 8;
  w = m.w;
  uint32_t bad = 0;
  if (w > MAXW) bad |= FLSGPU_BAD_BIT_WIDTH;
  if (c.n_packed && (m.off > c.n_packed || (size_t)w * Lanes<U>::N > c.n_packed - m.off))
    bad |= FLSGPU_BAD_OFFSET;
  vin = reinterpret_cast<const U *>(c.packed) + m.off;
  xf.base = m.base;
  if constexpr (std::is_same<T, float>::value) {
    if (m.fi > 9 || m.ei > 10) bad |= FLSGPU_BAD_PARAMETER_INDEX;
    if (!bad) {
      xf.fact = (uint32_t)(c.factors ? reinterpret_cast<const int32_t *>(c.factors)[m.fi]
                                     : c_f32_fact[m.fi]);
      xf.frac = c.fractions ? reinterpret_cast<const float *>(c.fractions)[m.ei] : c_f32_frac[m.ei];
    }
  } else if constexpr (std::is_same<T, double>::value) {
    if (m.fi > 18 || m.ei > 20) bad |= FLSGPU_BAD_PARAMETER_INDEX;
    if (!bad) {
      xf.fact = (uint64_t)(c.factors ? reinterpret_cast<const int64_t *>(c.factors)[m.fi]
                                     : c_f64_fact[m.fi]);
      xf.frac = c.fractions ? reinterpret_cast<const double *>(c.fractions)[m.ei] : c_f64_frac[m.ei];
    }
  }
  if (bad) {
    if (lane == 0) flag_status(d_status, bad);
    return false;
  }
  return true;
}

template <typename T, int KIND>
__device__ __forceinline__ bool vector_setup(const ColumnParams &c, uint32_t *d_status, size_t vi,
                                             int lane, const typename UintOf<T>::U *&vin, int &w,
                                             typename XformOf<T, KIND>::type &xf) {
  return setup_from_meta<T, KIND>(c, d_status, load_meta<T, KIND>(c, vi), lane, vin, w, xf);
}

// Asks L2 to fetch the packed lines (w lines of 128 B) of the next vector.
__device__ __forceinline__ void prefetch_packed(const void *vin, int w, int t) {
  const char *p = reinterpret_cast<const char *>(vin);
  for (int j = t; j < w; j += 32) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + 128 * j));
}

// Decodes the calling thread's 32 values of a vector; put(idx, value) with
// idx the position inside the vector, called in ascending value order.
// Kernel variant bits (chosen per type and width by the autotuner):
constexpr int VAR_STCS = 2;      // streaming (evict-first) output stores
constexpr int VAR_LD32 = 4;      // 64-bit lanes: 32-bit word loads (fewer live registers)
constexpr int VAR_MINB2 = 8;     // register cap for two resident blocks per SM
constexpr int VAR_CHUNK = 16;    // 64-bit lanes: decode half-lanes in two runs of 16
constexpr int VAR_AUTO = 32;     // per-width policy from autotune_table.h
constexpr int VAR_PAIR = 64;     // decode two same-width vectors per warp step (policy bit)
constexpr int VAR_NOPAIR = 128;  // kernel variant: never pair
constexpr int VAR_MINB4 = 256;   // kernel variant: 32-bit lanes capped for four blocks per SM
constexpr int VAR_OCC = 512;     // kernel variant: registers capped for twice the resident blocks
constexpr int VAR_MINB3 = 1024;  // kernel variant: registers capped for three resident blocks
constexpr int VAR_DEFAULT = VAR_AUTO;

// Policy bits in force for width W under kernel variant VAR.
// The register-capped variant (VAR_OCC) decodes wide 64-bit half-lanes in
// two runs of 16 values so that they fit its register budget.
template <typename U, int VAR> __host__ __device__ constexpr int policy_of(int W) {
  int pol = VAR;
  if constexpr ((VAR & VAR_AUTO) != 0) pol = sizeof(U) == 8 ? tuned::kPolicy64[W] : tuned::kPolicy32[W];
  if ((VAR & VAR_OCC) != 0 && sizeof(U) == 8 && W > 24) pol |= VAR_CHUNK;
  return pol;
}

// Widths decoded two vectors at a time (both vectors' loads in flight before
// either is unpacked): the low widths, whose code leaves most of the
// register allocation of the widest cases unused.
template <typename U, int VAR> __host__ __device__ constexpr unsigned long long pair_mask() {
  unsigned long long m = 0;
  if (VAR & VAR_NOPAIR) return 0;
  for (int w = 0; w <= (int)(sizeof(U) * 8) && w < 64; ++w)
    if (policy_of<U, VAR>(w) & VAR_PAIR) m |= 1ull << w;
  return m;
}

template <typename T, int VAR = VAR_DEFAULT, class X, class Put>
__device__ __forceinline__ void decode_values(const typename UintOf<T>::U *vin, int w, int t,
                                              const X &xf, Put &&put) {
  using U = typename UintOf<T>::U;
  if constexpr (sizeof(U) == 4) {
    switch_width32(w, [&](auto wc) {
      constexpr int W = decltype(wc)::value;
      constexpr int P = policy_of<U, VAR>(W);
      uint32_t wr[W > 0 ? W : 1];
      load_lane32<W>(vin, t, wr);
      unpack_lane32<W>(wr, [&](int k, uint32_t u) { put(t + 32 * k, xf(u), IntC<P>{}); });
    });
  } else {
    const int lane = t & 15, half = t >> 4;
    switch_width64(w, [&](auto wc) {
      constexpr int W = decltype(wc)::value;
      constexpr int P = policy_of<U, VAR>(W);
      if constexpr ((P & VAR_CHUNK) != 0 && W > 8) {
        decode_half64_chunked<W>(vin, lane, half, [&](int k, uint64_t u) {
          put(lane + 16 * (32 * half + k), xf(u), IntC<P>{});
        });
        return;
      }
      uint32_t wr[W > 0 ? W : 1];
      if constexpr ((P & VAR_LD32) != 0)
        load_half64_w32<W>(vin, lane, half, wr);
      else
        load_half64<W>(vin, lane, half, wr);
      unpack_half64<W>(wr, [&](int k, uint64_t u) {
        put(lane + 16 * (32 * half + k), xf(u), IntC<P>{});
      });
    });
  }
}

// Two vectors of the same width W: both vectors' packed words are loaded
// before either is unpacked.  Only called for widths in pair_mask.
template <typename T, int VAR, class X, class PutA, class PutB>
__device__ __forceinline__ void decode_pair(const typename UintOf<T>::U *va,
                                            const typename UintOf<T>::U *vb, int w, int t,
                                            const X &xa, const X &xb, PutA &&pa, PutB &&pb) {
  using U = typename UintOf<T>::U;
  constexpr unsigned long long PM = pair_mask<U, VAR>();
  if constexpr (sizeof(U) == 4) {
    switch_width32(w, [&](auto wc) {
      constexpr int W = decltype(wc)::value;
      if constexpr (W < 64 && ((PM >> W) & 1)) {
        constexpr int P = policy_of<U, VAR>(W);
        uint32_t wa[W > 0 ? W : 1], wb[W > 0 ? W : 1];
        load_lane32<W>(va, t, wa);
        load_lane32<W>(vb, t, wb);
        unpack_lane32<W>(wa, [&](int k, uint32_t u) { pa(t + 32 * k, xa(u), IntC<P>{}); });
        unpack_lane32<W>(wb, [&](int k, uint32_t u) { pb(t + 32 * k, xb(u), IntC<P>{}); });
      }
    });
  } else {
    const int lane = t & 15, half = t >> 4;
    switch_width64(w, [&](auto wc) {
      constexpr int W = decltype(wc)::value;
      if constexpr (W < 64 && ((PM >> W) & 1)) {
        constexpr int P = policy_of<U, VAR>(W);
        uint32_t wa[W > 0 ? W : 1], wb[W > 0 ? W : 1];
        load_half64<W>(va, lane, half, wa);
        load_half64<W>(vb, lane, half, wb);
        unpack_half64<W>(wa, [&](int k, uint64_t u) {
          pa(lane + 16 * (32 * half + k), xa(u), IntC<P>{});
        });
        unpack_half64<W>(wb, [&](int k, uint64_t u) {
          pb(lane + 16 * (32 * half + k), xb(u), IntC<P>{});
        });
      }
    });
  }
}

// Writes exceptions [from, cnt) of a vector (positions pos[i], values
// exc[i], both already offset to the vector's first exception) through
// write(position, value), four rounds of 32 at a time: every load of a
// batch is issued before its stores, so a vector with many exceptions waits
// one load latency per 128 of them instead of one per 32 (the stores may
// alias the loads as far as the compiler knows, so it cannot reorder them
// itself).  Returns true when a position was out of range (not written).
template <typename T, class Write>
__device__ __forceinline__ bool patch_batched(const uint16_t *pos, const T *exc, uint32_t from,
                                              uint32_t cnt, int t, Write &&write) {
  bool bad = false;
  for (uint32_t i0 = from; i0 < cnt; i0 += 128) {
    uint32_t ps[4];
    T ev[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t i = i0 + 32u * u + (uint32_t)t;
      ps[u] = i < cnt ? (uint32_t)pos[i] : 0xFFFFFFFFu;
      ev[u] = i < cnt ? exc[i] : T(0);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (ps[u] == 0xFFFFFFFFu) continue;
      if (ps[u] < (uint32_t)VEC)
        write(ps[u], ev[u]);
      else
        bad = true;
    }
  }
  return bad;
}

// Exceptions of vector vi (decoder::patch_exceptions, src/alp/decoder.hpp:
// 137-145): count = counts[vi] (ALPColumn) or the u16 sum of the per-lane
// counts (ALPExtendedColumn, as alp::decode reconstructs it,
// alp-bindings.cu:238-242).  Positions of a vector are distinct, so the
// warp writes them in parallel.
template <typename T, int KIND, class Write>
__device__ __forceinline__ void patch_vector(const ColumnParams &c, uint32_t *d_status, size_t vi,
                                             int t, Write &&write) {
  using U = typename UintOf<T>::U;
  constexpr int NL = Lanes<U>::N;
  uint32_t cnt;
  if constexpr (KIND == K_ALP) {
    cnt = c.counts[vi];
  } else {
    uint32_t lc = (t < NL) ? (uint32_t)(c.oc[vi * NL + t] >> 10) : 0u;
    cnt = __reduce_add_sync(0xffffffffu, lc) & 0xFFFFu;
  }
  const size_t eo = c.exc_offs[vi];
  const T *exc = reinterpret_cast<const T *>(c.exc);
  const bool bad = patch_batched<T>(c.pos + eo, exc + eo, 0, cnt, t, write);
  if (__any_sync(0xffffffffu, bad) && t == 0) flag_status(d_status, FLSGPU_BAD_EXCEPTION);
}

template <typename T, int T_VAR> __device__ __forceinline__ void store_out(T *p, T v) {
  if constexpr ((T_VAR & VAR_STCS) != 0)
    __stcs(p, v);
  else
    *p = v;
}

// Resident blocks per SM the register allocation must allow: the decode
// loop is latency-bound at low widths, so occupancy matters more than
// keeping every packed word of the widest cases in registers.
template <typename T, int VAR> constexpr int min_blocks() {
  constexpr int base = sizeof(T) == 4 ? 2 : 1;
  return (VAR & VAR_MINB4) ? 4 : (VAR & VAR_MINB3) ? 3 : (VAR & VAR_MINB2) ? 2 : (VAR & VAR_OCC) ? 2 * base : base;
}

__device__ __forceinline__ bool prefetch_width(const KernelParams &p, int w) {
  return w < 128 && ((p.prefetch[w >> 6] >> (w & 63)) & 1);
}

// Decodes one vector into the output (row order), then patches its
// exceptions for ALP columns.
template <typename T, int KIND, int VAR>
__device__ __forceinline__ void store_one(const KernelParams &p, size_t vi, const Meta<T> &m,
                                          int t) {
  using U = typename UintOf<T>::U;
  using X = typename XformOf<T, KIND>::type;
  constexpr bool IS_ALP = (KIND == K_ALP || KIND == K_ALPX);
  const ColumnParams &c = p.c;
  const U *vin;
  int w;
  X xf;
  if (!setup_from_meta<T, KIND>(c, p.d_status, m, t, vin, w, xf)) return;
  const size_t vbase = vi * VEC;
  const size_t rem = c.n_values - vbase;
  const int lim = rem < (size_t)VEC ? (int)rem : VEC;
  T *out = reinterpret_cast<T *>(p.out) + vbase;
  // ALPColumn: the vector's first 32 exceptions (position, value) are loaded
  // before the decode, so their latency overlaps the packed words' instead
  // of following the row stores.
  [[maybe_unused]] uint32_t p0 = VEC;
  [[maybe_unused]] T e0 = T(0);
  [[maybe_unused]] const bool pre =
      (KIND == K_ALP && c.patch && c.counts) || (KIND == K_ALPX && c.patch && c.oc);
  [[maybe_unused]] uint32_t ecnt = 0;
  if constexpr (KIND == K_ALP || KIND == K_ALPX) {
    if constexpr (KIND == K_ALP)
      ecnt = m.ecnt;
    else
      ecnt = __reduce_add_sync(0xffffffffu, m.ecnt >> 10) & 0xFFFFu;
    if (pre && (uint32_t)t < ecnt) {
      p0 = c.pos[m.eo + t];
      e0 = reinterpret_cast<const T *>(c.exc)[m.eo + t];
    }
  }
  if (lim == VEC) {
    decode_values<T, VAR>(vin, w, t, xf, [&](int idx, T v, auto pc) {
      store_out<T, decltype(pc)::value>(out + idx, v);
    });
  } else {
    decode_values<T, VAR>(vin, w, t, xf, [&](int idx, T v, auto pc) {
      if (idx < lim) store_out<T, decltype(pc)::value>(out + idx, v);
    });
  }
  if constexpr (KIND == K_ALP || KIND == K_ALPX) {
    if (pre) {
      __syncwarp();
      bool bad = (uint32_t)t < ecnt && p0 >= VEC;
      if ((int)p0 < lim) out[p0] = e0;
      const T *exc = reinterpret_cast<const T *>(c.exc);
      bad |= patch_batched<T>(c.pos + m.eo, exc + m.eo, 32, ecnt, t, [&](uint32_t ps, T e) {
        if ((int)ps < lim) out[ps] = e;
      });
      if (__any_sync(0xffffffffu, bad) && t == 0) flag_status(p.d_status, FLSGPU_BAD_EXCEPTION);
      return;
    }
  }
  if constexpr (IS_ALP) {
    if (c.patch) {
      __syncwarp();
      patch_vector<T, KIND>(c, p.d_status, vi, t, [&](int ps, T e) {
        if (ps < lim) out[ps] = e;
      });
    }
  }
}

// Full decompression.  The warp walks its vectors with a stride of the
// grid's warp count, keeping the metadata of the next one or two vectors in
// flight; two consecutive vectors of the same low width are decoded as a
// pair (decode_pair).
template <typename T, int KIND, int VAR = VAR_DEFAULT>
__global__ void __launch_bounds__(256, min_blocks<T, VAR>()) k_store(const KernelParams p) {
  using U = typename UintOf<T>::U;
  using X = typename XformOf<T, KIND>::type;
  constexpr bool IS_ALP = (KIND == K_ALP || KIND == K_ALPX);
  constexpr unsigned long long PM = pair_mask<U, VAR>();
  const int t = threadIdx.x & 31;
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const ColumnParams &c = p.c;
  const size_t n = c.n_vecs;
  T *const out_all = reinterpret_cast<T *>(p.out);
  (void)out_all;

  Meta<T> ma, mb;
  size_t vi = gw;
  if (vi < n) ma = load_meta<T, KIND>(c, vi, t);
  bool hb = vi + nw < n;
  if (hb) mb = load_meta<T, KIND>(c, vi + nw, t);
  while (vi < n) {
    // pair when both vectors are full and share a width marked for pairing
    const bool pair = PM != 0 && hb && ma.w == mb.w && ma.w < 64 && ((PM >> ma.w) & 1) &&
                      (vi + nw) * VEC + VEC <= c.n_values;
    Meta<T> na, nb;
    bool hnb;
    if (pair) {
      if (vi + 2 * nw < n) na = load_meta<T, KIND>(c, vi + 2 * nw, t);
      hnb = vi + 3 * nw < n;
      if (hnb) nb = load_meta<T, KIND>(c, vi + 3 * nw, t);
    } else {
      na = mb;
      hnb = vi + 2 * nw < n;
      if (hnb) nb = load_meta<T, KIND>(c, vi + 2 * nw, t);
    }
    {
      const size_t vn = vi + (pair ? 2 : 1) * nw;
      if (vn < n && na.w <= (int)(sizeof(U) * 8) && prefetch_width(p, na.w))
        prefetch_packed(reinterpret_cast<const U *>(c.packed) + na.off, na.w, t);
    }
    if (pair) {
      const U *va, *vb;
      int wa, wb;
      X xa, xb;
      const bool oka = setup_from_meta<T, KIND>(c, p.d_status, ma, t, va, wa, xa);
      const bool okb = setup_from_meta<T, KIND>(c, p.d_status, mb, t, vb, wb, xb);
      const size_t vj = vi + nw;
      if (oka && okb) {
        T *outa = out_all + vi * VEC, *outb = out_all + vj * VEC;
        decode_pair<T, VAR>(
            va, vb, wa, t, xa, xb,
            [&](int idx, T v, auto pc) { store_out<T, decltype(pc)::value>(outa + idx, v); },
            [&](int idx, T v, auto pc) { store_out<T, decltype(pc)::value>(outb + idx, v); });
        if constexpr (IS_ALP) {
          if (c.patch) {
            __syncwarp();
            patch_vector<T, KIND>(c, p.d_status, vi, t, [&](int ps, T e) { outa[ps] = e; });
            patch_vector<T, KIND>(c, p.d_status, vj, t, [&](int ps, T e) { outb[ps] = e; });
          }
        }
      } else {
        if (oka) store_one<T, KIND, VAR>(p, vi, ma, t);
        if (okb) store_one<T, KIND, VAR>(p, vj, mb, t);
      }
      vi += 2 * nw;
    } else {
      store_one<T, KIND, VAR>(p, vi, ma, t);
      vi += nw;
    }
    ma = na;
    mb = nb;
    hb = hnb;
  }
}

// ---- integer sums: the sum of a thread's 32 packed values ------------------
// A thread's 32 values of width W are the stream of its W words w[0..W-1]
// (lane t of a 32-bit vector, or half-lane t / 16 of lane t % 16 of a
// 64-bit one after words_of_half64): value k is stream bits [kW, kW + W).
// Bit o of word j is therefore bit (32 j + o) mod W of its value, and the
// sum of the 32 values is sum over j, b of popc(w[j] & M(W, j, b)) << b,
// where M(W, j, b) marks the bits of word j at value bit b -- W * W
// popcounts instead of 32 unpacks and adds, fewer instructions up to
// kPopW.  Up to 26 bits the 32 values sum within 32 bits.
constexpr int kPopW = 4;
constexpr int kSum32W = 26;

__host__ __device__ constexpr uint32_t plane_mask(int W, int j, int b) {
  uint32_t m = 0;
  for (int o = 0; o < 32; ++o)
    if ((32 * j + o) % W == b) m |= 1u << o;
  return m;
}

template <int W, int J, int B>
__device__ __forceinline__ uint32_t plane_sum(const uint32_t *w) {
  if constexpr (J == W) {
    return 0u;
  } else if constexpr (B == W) {
    return plane_sum<W, J + 1, 0>(w);
  } else {
    constexpr uint32_t M = plane_mask(W, J, B);
    return ((uint32_t)__popc(w[J] & M) << B) + plane_sum<W, J, B + 1>(w);
  }
}

// Sum of the calling thread's 32 values u (without the base) of a vector
// of width w <= kSum32W.
template <typename U>
__device__ __forceinline__ uint32_t thread_sum_narrow(const U *vin, int w, int t) {
  uint32_t s = 0;
  switch_width26(w, [&](auto wc) {
    constexpr int W = decltype(wc)::value;
    if constexpr (W > 0) {
      uint32_t wr[W];
      if constexpr (sizeof(U) == 4)
        load_lane32<W>(vin, t, wr);
      else
        load_half64<W>(vin, t & 15, t >> 4, wr);
      if constexpr (W <= kPopW)
        s = plane_sum<W, 0, 0>(wr);
      else
        unpack_lane32<W>(wr, [&](int, uint32_t u) { s += u; });
    }
  });
  return s;
}

template <typename T, int KIND, int SINK, int VAR = VAR_DEFAULT>
__global__ void __launch_bounds__(256, min_blocks<T, VAR>()) k_column(const KernelParams p) {
  using U = typename UintOf<T>::U;
  using X = typename XformOf<T, KIND>::type;
  constexpr bool IS_ALP = (KIND == K_ALP || KIND == K_ALPX);
  // ALP sums / scans stage the patched vector in shared memory.
  constexpr bool STAGE = IS_ALP && SINK != S_STORE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sbuf = reinterpret_cast<T *>(smem_raw) + (threadIdx.x >> 5) * (STAGE ? VEC : 0);

  const int t = threadIdx.x & 31;
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const ColumnParams &c = p.c;
  const T magic = from_bits<T>(p.magic);

  uint64_t acc_u = 0;
  bool flag = false;

  Meta<T> meta;
  if (gw < c.n_vecs) meta = load_meta<T, KIND>(c, gw);
  for (size_t vi = gw; vi < c.n_vecs; vi += nw) {
    const U *vin;
    int w;
    X xf;
    const Meta<T> cur = meta;
    if (vi + nw < c.n_vecs) {
      meta = load_meta<T, KIND>(c, vi + nw);
      bool pf = meta.w <= (int)(sizeof(U) * 8) && prefetch_width(p, meta.w);
      if constexpr (SINK == S_QUERY && !IS_ALP)  // not for a vector the range test skips
        pf = pf && (meta.w == (int)(sizeof(U) * 8) || (((U)magic - meta.base) >> meta.w) == 0);
      if (pf) prefetch_packed(reinterpret_cast<const U *>(c.packed) + meta.off, meta.w, t);
    }
    if (!setup_from_meta<T, KIND>(c, p.d_status, cur, t, vin, w, xf)) {
      // a rejected vector (status flag raised) adds +0.0: its slot of the
      // fixed tree gets a defined value, never what the buffer held before
      if constexpr (STAGE && SINK == S_SUM) {
        if (t == 0) p.partials[vi] = 0.0;
      }
      continue;
    }
    const size_t vbase = vi * VEC;
    const size_t rem = c.n_values - vbase;
    const int lim = rem < (size_t)VEC ? (int)rem : VEC;

    if constexpr (SINK == S_STORE) {
      T *out = reinterpret_cast<T *>(p.out) + vbase;
      if (lim == VEC) {
        decode_values<T, VAR>(vin, w, t, xf, [&](int idx, T v, auto pc) {
          store_out<T, decltype(pc)::value>(out + idx, v);
        });
      } else {
        decode_values<T, VAR>(vin, w, t, xf, [&](int idx, T v, auto pc) {
          if (idx < lim) store_out<T, decltype(pc)::value>(out + idx, v);
        });
      }
      if constexpr (IS_ALP) {
        if (c.patch) {
          __syncwarp();
          patch_vector<T, KIND>(c, p.d_status, vi, t, [&](int ps, T e) {
            if (ps < lim) out[ps] = e;
          });
        }
      }
    } else if constexpr (STAGE) {
      decode_values<T>(vin, w, t, xf, [&](int idx, T v, auto...) { sbuf[idx] = v; });
      __syncwarp();
      if (c.patch) patch_vector<T, KIND>(c, p.d_status, vi, t, [&](int ps, T e) { sbuf[ps] = e; });
      __syncwarp();
      if constexpr (SINK == S_SUM) {
        // fixed tree: per-thread ascending sum, warp butterfly
        double acc = 0.0;
        if constexpr (sizeof(T) == 8) {
          const int lane = t & 15, half = t >> 4;
#pragma unroll 8
          for (int k = 0; k < 32; ++k) {
            const int idx = lane + 16 * (32 * half + k);
            if (idx < lim) acc = __dadd_rn(acc, (double)sbuf[idx]);
          }
        }
#pragma unroll
        for (int s = 16; s >= 1; s >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, s));
        if (t == 0) p.partials[vi] = acc;
      } else if constexpr (SINK == S_QUERY) {
        for (int idx = t; idx < lim; idx += 32) flag |= (sbuf[idx] == magic);
      } else if constexpr (SINK == S_ALLEQ) {
        bool all = true;
        constexpr int NL = Lanes<U>::N;
        if (t < NL)
          for (int k = 0; k < (int)(sizeof(U) * 8); ++k) {
            const int idx = t + NL * k;
            if (idx < lim) all &= (sbuf[idx] == magic);
          }
        flag |= (t < NL) && all;
      }
      __syncwarp();
    } else {
      // register sinks for integer columns
      if constexpr (SINK == S_SUM) {
        // sum of (u + base): with 64-bit lanes the accumulator wraps as the
        // values do, so the base enters once per vector (1024 * base); with
        // 32-bit lanes only when no value of the vector wraps (base + 2^w - 1
        // < 2^32).  Full vectors take no per-value bound test.
        const U base = xf.base;
        const bool once = sizeof(U) == 8 || (uint64_t)base + ((1ull << w) - 1ull) < (1ull << 32);
        if (lim == VEC && once) {
          uint64_t sv = 0;
          if (w <= kSum32W)
            sv = thread_sum_narrow<U>(vin, w, t);
          else
            decode_values<T, VAR>(vin, w, t, XInt<U>{U(0)},
                                  [&](int, T v, auto...) { sv += (uint64_t)v; });
          acc_u += sv + (t == 0 ? (uint64_t)base * (uint64_t)VEC : 0ull);
        } else {
          decode_values<T, VAR>(vin, w, t, xf, [&](int idx, T v, auto...) {
            if (idx < lim) acc_u += (uint64_t)v;
          });
        }
      } else if constexpr (SINK == S_QUERY) {
        // a vector of width w holds (u + base) mod 2^bits with u < 2^w: it
        // can hold the magic value only if u = (magic - base) mod 2^bits is
        // below 2^w, so other vectors are decided on their metadata alone
        const U target = (U)magic - xf.base;
        if (w < (int)(sizeof(U) * 8) && (target >> w) != 0) continue;
        if (lim == VEC) {
          decode_values<T, VAR>(vin, w, t, XInt<U>{U(0)},
                                [&](int, T v, auto...) { flag |= v == target; });
        } else {
          decode_values<T, VAR>(vin, w, t, XInt<U>{U(0)},
                                [&](int idx, T v, auto...) { flag |= (idx < lim) && (v == target); });
        }
      } else if constexpr (SINK == S_COMPUTE) {
        const T zero = (T)p.runtime_zero;
        const uint32_t nrep = p.n_rep;
        decode_values<T>(vin, w, t, xf, [&](int idx, T v, auto...) {
          // kernels::device::compute_column, src/engine/kernels.cuh:75-84
          for (uint32_t r = 0; r < nrep; ++r) {
            v *= (T)3;
            v <<= 3;
            v += (T)3;
            v >>= 3;
            v &= zero;
          }
          flag |= (idx < lim) && (v == (T)1);
        });
      } else if constexpr (SINK == S_ALLEQ) {
        bool all = true;
        decode_values<T>(vin, w, t, xf, [&](int idx, T v, auto...) { all &= (idx >= lim) || (v == magic); });
        if constexpr (sizeof(U) == 8) all = all && __shfl_xor_sync(0xffffffffu, all, 16);
        flag |= all;
      }
    }
  }

  if constexpr (SINK == S_SUM && !IS_ALP) {
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) acc_u += __shfl_xor_sync(0xffffffffu, acc_u, s);
    if (t == 0 && acc_u) atomicAdd(reinterpret_cast<unsigned long long *>(p.sum_u64),
                                   (unsigned long long)acc_u);
  }
  if constexpr (SINK == S_QUERY || SINK == S_COMPUTE || SINK == S_ALLEQ) {
    if (__any_sync(0xffffffffu, flag) && t == 0) *p.found = 1;
  }
}

// Pairwise tree over vector partials (stride doubling, aligned chunks of
// 2048): dst[b] = tree(src[2048 b .. 2048 b + 2047]).
static __global__ void __launch_bounds__(1024) k_pairwise_f64(const double *src, size_t n, double *dst) {
  __shared__ double s[2048];
  const size_t base = (size_t)blockIdx.x * 2048;
  const size_t m = std::min<size_t>(2048, n - base);
  for (int i = threadIdx.x; i < 2048; i += 1024) s[i] = (size_t)i < m ? src[base + i] : 0.0;
  __syncthreads();
  for (int st = 1; st < 2048; st <<= 1) {
    const int i = threadIdx.x * 2 * st;
    if (i < 2048 && (size_t)(i + st) < m) s[i] = __dadd_rn(s[i], s[i + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0) dst[blockIdx.x] = s[0];
}

// ---- host side ------------------------------------------------------------
// Host-side decode tuning (capi.cu): the kernel variant used under
// FLSGPU_VARIANT_AUTO per (value type, column kind), and the per-width L2
// prefetch masks per lane width; defaults from autotune_table.h, replaced
// by the autotuner through flsgpu_tuning_set_*.
int tuned_variant(int type, int kind);
void tuned_prefetch(int lane_bits, uint64_t out[2]);
template <typename T> constexpr int type_code() {
  return std::is_same<T, uint32_t>::value ? 0 : std::is_same<T, uint64_t>::value ? 1
       : std::is_same<T, float>::value ? 2 : 3;
}

// The staged decode of 64-bit lanes (staged.cuh).
template <typename T, int KIND> flsgpu_status launch_staged(const KernelParams &p, cudaStream_t s);

template <typename T, int KIND, int SINK> struct Launch {
  static constexpr bool STAGE = (KIND == K_ALP || KIND == K_ALPX) && SINK != S_STORE;
  static size_t smem() { return STAGE ? (size_t)8 * VEC * sizeof(T) : 0; }
  // Integer sums and scans hold no decoded values, only the packed words in
  // flight: their kernel is register-capped for more resident warps (wide
  // 64-bit half-lanes decode in two runs of 16), which multiplies the loads
  // each SM keeps in flight.
  static constexpr int COL_VAR =
      ((SINK == S_SUM || SINK == S_QUERY) && (KIND == K_BP || KIND == K_FFOR))
          ? (VAR_AUTO | VAR_OCC | (sizeof(T) == 8 && SINK == S_SUM ? VAR_MINB3 : 0))
          : VAR_DEFAULT;
  template <int V> static auto kernel() {
    if constexpr (SINK == S_STORE)
      return k_store<T, KIND, VAR_AUTO | V>;
    else
      return k_column<T, KIND, SINK, COL_VAR>;
  }
  template <int V> static int blocks_per_sm() {
    static int bps = 0;
    if (bps == 0) {
      auto kern = kernel<V>();
      if (smem() > 48 * 1024)
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem());
      int b = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, 256, smem());
      bps = b > 0 ? b : 1;
    }
    return bps;
  }
  template <int V> static flsgpu_status launch(const KernelParams &p, cudaStream_t s) {
    const unsigned grid = persistent_blocks(p.c.n_vecs, 8, blocks_per_sm<V>());
    kernel<V>()<<<grid, 256, smem(), s>>>(p);
    note_launch();
    return check_cuda(cudaGetLastError(), "decode launch");
  }
  // variant: FLSGPU_VARIANT_* (full decompression only; the fused sinks
  // have one kernel each)
  static flsgpu_status run(KernelParams p, cudaStream_t s, uint32_t variant = FLSGPU_VARIANT_AUTO) {
    if (p.c.n_vecs == 0) return FLSGPU_OK;
    tuned_prefetch((int)sizeof(T) * 8, p.prefetch);
    if constexpr (SINK == S_STORE) {
      if (variant == FLSGPU_VARIANT_AUTO) variant = (uint32_t)tuned_variant(type_code<T>(), KIND);
      if (variant == FLSGPU_VARIANT_OCCUPANCY) return launch<VAR_OCC>(p, s);
      if constexpr (sizeof(T) == 8) {
        if (variant == FLSGPU_VARIANT_STAGED) return launch_staged<T, KIND>(p, s);
      }
    }
    return launch<0>(p, s);
  }
};

static inline size_t vecs_of(size_t n_values) { return (n_values + VEC - 1) / VEC; }

static inline bool patch_enabled(const flsgpu_decode_opts *o) {
  return !o || (o->patcher != FLSGPU_PATCHER_NONE && o->patcher != FLSGPU_PATCHER_DUMMY);
}

static inline flsgpu_status check_opts(const flsgpu_decode_opts *o) {
  if (!o) return FLSGPU_OK;
  if (o->unpacker >= FLSGPU_UNPACKER_COUNT)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "unknown unpacker %u", o->unpacker);
  if (o->patcher >= FLSGPU_PATCHER_COUNT)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "unknown patcher %u", o->patcher);
  if (o->variant >= FLSGPU_VARIANT_COUNT)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "unknown variant %u", o->variant);
  if (o->unpack_n_vectors > 8 || o->unpack_n_values > 32)
    return set_error(FLSGPU_ERR_UNSUPPORTED, "unpack_n_vectors %u / unpack_n_values %u",
                     o->unpack_n_vectors, o->unpack_n_values);
  return FLSGPU_OK;
}

static inline flsgpu_status fill_bp(ColumnParams &c, const flsgpu_bp_column *bp, size_t n_values) {
  c.n_values = n_values;
  c.n_vecs = vecs_of(n_values);
  c.packed = bp->packed_array;
  c.bw = bp->bit_widths;
  c.offs = bp->vector_offsets;
  if (c.n_vecs && (!c.bw || !c.offs))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null bit_widths / vector_offsets");
  return FLSGPU_OK;
}

static inline flsgpu_status fill(ColumnParams &c, const flsgpu_bp_column *col, const flsgpu_decode_opts *o) {
  if (!col) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  c = ColumnParams{};
  c.n_packed = o ? o->n_packed_values : 0;
  return fill_bp(c, col, col->n_values);
}
static inline flsgpu_status fill(ColumnParams &c, const flsgpu_ffor_column *col, const flsgpu_decode_opts *o) {
  if (!col) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  c = ColumnParams{};
  c.n_packed = o ? o->n_packed_values : 0;
  flsgpu_status s = fill_bp(c, &col->bp, col->n_values);
  if (s) return s;
  c.bases = col->bases;
  if (c.n_vecs && !c.bases) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null bases");
  return FLSGPU_OK;
}
template <typename AC>
static flsgpu_status fill_alp(ColumnParams &c, const AC *col, const flsgpu_decode_opts *o) {
  if (!col) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  flsgpu_status s = fill(c, &col->ffor, o);
  if (s) return s;
  c.n_values = col->n_values;
  c.n_vecs = vecs_of(col->n_values);
  c.factors = col->factors;
  c.fractions = col->fractions;
  c.fac_idx = col->factor_indices;
  c.exp_idx = col->fraction_indices;
  c.exc_offs = col->exceptions_offsets;
  c.exc = col->exceptions;
  c.pos = col->positions;
  c.patch = patch_enabled(o) ? 1 : 0;
  if (c.n_vecs && (!c.fac_idx || !c.exp_idx))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null factor / fraction indices");
  return FLSGPU_OK;
}
static inline flsgpu_status fill(ColumnParams &c, const flsgpu_alp_column *col, const flsgpu_decode_opts *o) {
  flsgpu_status s = fill_alp(c, col, o);
  if (s) return s;
  c.counts = col->counts;
  if (c.patch && c.n_vecs && (!c.counts || !c.exc_offs))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null exception arrays");
  return FLSGPU_OK;
}
static inline flsgpu_status fill(ColumnParams &c, const flsgpu_alpx_column *col, const flsgpu_decode_opts *o) {
  flsgpu_status s = fill_alp(c, col, o);
  if (s) return s;
  c.oc = col->offsets_counts;
  if (c.patch && c.n_vecs && (!c.oc || !c.exc_offs))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null exception arrays");
  return FLSGPU_OK;
}

template <typename T> static bool aligned(const void *p) {
  return ((uintptr_t)p % sizeof(T)) == 0;
}

template <typename T, int KIND, typename Col>
static flsgpu_status decompress(const Col *col, T *d_out, const flsgpu_decode_opts *o,
                                flsgpu_stream stream) {
  flsgpu_status s = check_opts(o);
  if (s) return s;
  KernelParams p{};
  if ((s = fill(p.c, col, o))) return s;
  if (p.c.n_vecs == 0) return FLSGPU_OK;
  if (!d_out) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null output");
  if (!aligned<T>(d_out)) return set_error(FLSGPU_ERR_MISALIGNED, "output not aligned");
  p.d_status = o ? o->d_status : nullptr;
  p.out = d_out;
  return Launch<T, KIND, S_STORE>::run(p, (cudaStream_t)stream,
                                       o ? o->variant : (uint32_t)FLSGPU_VARIANT_AUTO);
}

template <typename T, int KIND, typename Col>
static flsgpu_status query(const Col *col, T magic, uint8_t *d_found, const flsgpu_decode_opts *o,
                           flsgpu_stream stream) {
  flsgpu_status s = check_opts(o);
  if (s) return s;
  KernelParams p{};
  if ((s = fill(p.c, col, o))) return s;
  if (!d_found) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null result");
  p.d_status = o ? o->d_status : nullptr;
  p.found = d_found;
  uint64_t bits = 0;
  memcpy(&bits, &magic, sizeof(T));
  p.magic = bits;
  return Launch<T, KIND, S_QUERY>::run(p, (cudaStream_t)stream);
}

template <typename T, typename Col>
static flsgpu_status sum_int(const Col *col, uint64_t *d_sum, const flsgpu_decode_opts *o,
                             flsgpu_stream stream) {
  flsgpu_status s = check_opts(o);
  if (s) return s;
  KernelParams p{};
  if ((s = fill(p.c, col, o))) return s;
  if (!d_sum) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null sum");
  if ((s = check_cuda(cudaMemsetAsync(d_sum, 0, sizeof(uint64_t), (cudaStream_t)stream),
                      "memset sum")))
    return s;
  p.d_status = o ? o->d_status : nullptr;
  p.sum_u64 = d_sum;
  return Launch<T, K_FFOR, S_SUM>::run(p, (cudaStream_t)stream);
}

// Reduces n partials (fixed pairwise tree) into *d_sum, using `tmp` (at
// least (n + 2047) / 2048 elements) as scratch.
static inline flsgpu_status pairwise_f64(double *partials, size_t n, double *tmp, double *d_sum,
                                  cudaStream_t stream) {
  if (n == 0) return check_cuda(cudaMemsetAsync(d_sum, 0, sizeof(double), stream), "memset");
  double *src = partials, *dst = tmp;
  while (n > 1) {
    const size_t nb = (n + 2047) / 2048;
    double *d = (nb == 1) ? d_sum : dst;
    k_pairwise_f64<<<(unsigned)nb, 1024, 0, stream>>>(src, n, d);
    note_launch();
    flsgpu_status s = check_cuda(cudaGetLastError(), "k_pairwise_f64");
    if (s) return s;
    if (nb == 1) return FLSGPU_OK;
    // ping-pong between the scratch area and the head of the partials
    double *nsrc = d;
    dst = (d == tmp) ? partials : tmp;
    src = nsrc;
    n = nb;
  }
  return check_cuda(cudaMemcpyAsync(d_sum, src, sizeof(double), cudaMemcpyDeviceToDevice, stream),
                    "copy sum");
}

template <int KIND, typename Col>
static flsgpu_status sum_f64(const Col *col, double *d_sum, double *d_partials,
                             const flsgpu_decode_opts *o, flsgpu_stream stream) {
  flsgpu_status s = check_opts(o);
  if (s) return s;
  KernelParams p{};
  if ((s = fill(p.c, col, o))) return s;
  if (!d_sum || (p.c.n_vecs && !d_partials))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null sum / partials");
  p.d_status = o ? o->d_status : nullptr;
  p.partials = d_partials;
  if ((s = Launch<double, KIND, S_SUM>::run(p, (cudaStream_t)stream))) return s;
  return pairwise_f64(d_partials, p.c.n_vecs, d_partials + p.c.n_vecs, d_sum,
                      (cudaStream_t)stream);
}

// ---- multi-column conjunctive scan ----------------------------------------
struct MultiParams {
  ColumnParams c[16];
  uint32_t n_cols;
  uint64_t value;
  uint8_t *out;
  uint32_t *d_status;
};

// multi_column::query_multi_column (src/generated-bindings/
// multi-column-device-kernels.cuh:11-439): a thread keeps
// all_columns_equal &= (reg[c] == reg[c-1]) and reg[0] == value over its
// lane in every column, which is "every value of the lane equals value in
// every column"; *out = 1 when some lane of some vector satisfies it.
template <typename T, int KIND>
__global__ void __launch_bounds__(256) k_multi(const MultiParams mp) {
  using U = typename UintOf<T>::U;
  using X = typename XformOf<T, KIND>::type;
  constexpr bool IS_ALP = (KIND == K_ALP || KIND == K_ALPX);
  constexpr int NL = Lanes<U>::N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sbuf = reinterpret_cast<T *>(smem_raw) + (threadIdx.x >> 5) * (IS_ALP ? VEC : 0);
  const int t = threadIdx.x & 31;
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const T value = from_bits<T>(mp.value);
  const size_t n_vecs = mp.c[0].n_vecs;
  bool flag = false;
  for (size_t vi = gw; vi < n_vecs; vi += nw) {
    bool all = true;
    for (uint32_t ci = 0; ci < mp.n_cols; ++ci) {
      const ColumnParams &c = mp.c[ci];
      const U *vin;
      int w;
      X xf;
      if (!vector_setup<T, KIND>(c, mp.d_status, vi, t, vin, w, xf)) {
        all = false;
        continue;
      }
      [[maybe_unused]] U target = 0;
      if constexpr (!IS_ALP) {
        // the vector holds (u + base) mod 2^bits with u < 2^w: no lane can
        // equal the value throughout unless (value - base) mod 2^bits < 2^w
        target = (U)value - xf.base;
        if (w < (int)(sizeof(U) * 8) && (target >> w) != 0) all = false;
      }
      // once no lane of the warp can qualify, the vector's remaining columns
      // are only validated (their metadata checks still raise the status)
      if (!__any_sync(0xffffffffu, all && (!IS_ALP || t < NL))) continue;
      const size_t rem = c.n_values - vi * VEC;
      const int lim = rem < (size_t)VEC ? (int)rem : VEC;
      if constexpr (IS_ALP) {
        decode_values<T>(vin, w, t, xf, [&](int idx, T v, auto...) { sbuf[idx] = v; });
        __syncwarp();
        if (c.patch) patch_vector<T, KIND>(c, mp.d_status, vi, t, [&](int ps, T e) { sbuf[ps] = e; });
        __syncwarp();
        if (t < NL)
          for (int k = 0; k < (int)(sizeof(U) * 8); ++k) {
            const int idx = t + NL * k;
            all &= (idx >= lim) || (sbuf[idx] == value);
          }
        __syncwarp();
      } else {
        decode_values<T>(vin, w, t, XInt<U>{U(0)},
                         [&](int idx, T v, auto...) { all &= (idx >= lim) || (v == target); });
      }
    }
    if constexpr (IS_ALP) {
      flag |= (t < NL) && all;
    } else {
      if constexpr (sizeof(U) == 8) all = all && __shfl_xor_sync(0xffffffffu, all, 16);
      flag |= all;
    }
  }
  if (__any_sync(0xffffffffu, flag) && t == 0) *mp.out = 1;
}

template <typename T, int KIND, typename Col>
static flsgpu_status multi(const Col *cols, uint32_t n, T value, uint8_t *d_out,
                           const flsgpu_decode_opts *o, flsgpu_stream stream) {
  flsgpu_status s = check_opts(o);
  if (s) return s;
  if (!cols || n == 0 || n > 16 || !d_out)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "bad multi-column arguments (n=%u)", n);
  MultiParams mp{};
  for (uint32_t i = 0; i < n; ++i) {
    if ((s = fill(mp.c[i], &cols[i], o))) return s;
    if (mp.c[i].n_vecs != mp.c[0].n_vecs)
      return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "columns differ in length");
  }
  if (mp.c[0].n_vecs == 0) return FLSGPU_OK;
  mp.n_cols = n;
  memcpy(&mp.value, &value, sizeof(T));
  mp.out = d_out;
  mp.d_status = o ? o->d_status : nullptr;
  constexpr bool IS_ALP = (KIND == K_ALP || KIND == K_ALPX);
  const size_t smem = IS_ALP ? (size_t)8 * VEC * sizeof(T) : 0;
  static int bps = 0;
  auto kern = k_multi<T, KIND>;
  if (bps == 0) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, 256, smem);
    bps = b > 0 ? b : 1;
  }
  const unsigned grid = persistent_blocks(mp.c[0].n_vecs, 8, bps);
  kern<<<grid, 256, smem, (cudaStream_t)stream>>>(mp);
  note_launch();
  return check_cuda(cudaGetLastError(), "k_multi launch");
}

template <typename T, typename Col>
static flsgpu_status compute(const Col *col, uint32_t n_rep, uint8_t *d_out,
                             const flsgpu_decode_opts *o, flsgpu_stream stream) {
  flsgpu_status s = check_opts(o);
  if (s) return s;
  KernelParams p{};
  if ((s = fill(p.c, col, o))) return s;
  if (!d_out) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null result");
  p.d_status = o ? o->d_status : nullptr;
  p.found = d_out;
  p.n_rep = n_rep;
  p.runtime_zero = 0;
  return Launch<T, K_FFOR, S_COMPUTE>::run(p, (cudaStream_t)stream);
}

}  // namespace flsb200

#include "staged.cuh"
