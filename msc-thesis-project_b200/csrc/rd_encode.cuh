// rd_encode.cuh -- device side of the GPU ALP-RD encoder (the reference has
// CPU code only, src/alp/rd.hpp):
//   find_best_dictionary (rd.hpp:83-98): try cutting 1..16 bits off the top
//     of the values' bit patterns; per cut the left parts of the sample are
//     counted, the 8 most frequent form the dictionary, the others are
//     exceptions, and the cut with the smallest estimated bits per value
//     (rd.hpp:18-25: right width + left width + 32 bits per exception / the
//     sample size) wins, the first one scanned on ties;
//   build_left_parts_dictionary (rd.hpp:28-81): left width
//     max(1, ceil(log2(dictionary size)));
//   encode (rd.hpp:103-140): right part = low right_bw bits, left part =
//     its dictionary index, or an exception (left part + position) when the
//     left part is not in the dictionary.
//
// One warp works on one sample (a rowgroup's first-level sample, at most
// kRDMaxSamples values, or a vector's 32 samples).  The sample is first
// sorted (rank sort in shared memory); because a left part is the value
// shifted right, equal left parts are then contiguous for every cut, and a
// run's length (binary search for its end) is the left part's count.  The
// dictionary is picked by 8 rounds of a warp maximum over (count, -start):
// the most frequent left part first, the smaller one among equal counts
// (the reference orders ties by unordered_map iteration; the dictionary is
// the same set whenever the 8th and 9th counts differ).
#pragma once

#include "common.cuh"

namespace flsb200 {

template <typename T> struct RDT;
template <> struct RDT<double> { using U = uint64_t; static constexpr int TB = 64; };
template <> struct RDT<float> { using U = uint32_t; static constexpr int TB = 32; };

constexpr int kRDMaxSamples = 320;  // a rowgroup of up to 100 vectors: 9 sampled vectors x 32
constexpr int kRDCuts = 16;         // config::CUTTING_LIMIT
constexpr int kRDDict = 8;          // config::MAX_RD_DICTIONARY_SIZE

// The chosen cut of one sample: right width, left width, dictionary size,
// and entry r of the dictionary on lane r (r < dsize; 0 elsewhere).
struct RDChoice {
  int rbw, lbw, dsize;
  uint32_t entry;
};

// srt[0..ns) = smp[0..ns) in ascending unsigned order (ranks by value, then
// index, so equal values keep distinct slots).
template <typename U>
__device__ __forceinline__ void rd_rank_sort(const U *smp, int ns, U *srt, int t) {
  for (int i = t; i < ns; i += 32) {
    const U x = smp[i];
    int r = 0;
    for (int j = 0; j < ns; ++j) {
      const U y = smp[j];
      r += (y < x) || (y == x && j < i);
    }
    srt[r] = x;
  }
  __syncwarp();
}

// build_left_parts_dictionary for one cut of the sorted sample: returns the
// estimated bits per value; *dsize, *lbw and (lane r) *entry receive the
// dictionary when the pointers are given.
template <typename U, int NSMAX = kRDMaxSamples>
__device__ double rd_cut(const U *srt, int ns, int rbw, int t, int *dsize_out, int *lbw_out,
                         uint32_t *entry) {
  constexpr int MAXI = (NSMAX + 31) / 32;
  // per lane: its run heads j = t + 32 i as (count << 12) | (4095 - j)
  uint32_t code[MAXI];
#pragma unroll
  for (int i = 0; i < MAXI; ++i) {
    const int j = t + 32 * i;
    code[i] = 0;
    if (j < ns) {
      const U key = srt[j] >> rbw;
      if (j == 0 || (srt[j - 1] >> rbw) != key) {
        int lo = j + 1, hi = ns;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if ((srt[mid] >> rbw) > key)
            hi = mid;
          else
            lo = mid + 1;
        }
        code[i] = ((uint32_t)(lo - j) << 12) | (uint32_t)(4095 - j);
      }
    }
  }
  int d = 0, in_dict = 0;
  uint32_t ent = 0;
  for (; d < kRDDict; ++d) {
    uint32_t best = 0;
#pragma unroll
    for (int i = 0; i < MAXI; ++i) best = code[i] > best ? code[i] : best;
    best = __reduce_max_sync(0xffffffffu, best);
    if (best == 0) break;
    const int j = 4095 - (int)(best & 4095u);
    in_dict += (int)(best >> 12);
#pragma unroll
    for (int i = 0; i < MAXI; ++i)
      if ((j & 31) == t && i == (j >> 5)) code[i] = 0;
    if (t == d) ent = (uint32_t)(srt[j] >> rbw);
  }
  // max(1, ceil(log2(d))) for d = 1..8
  const int lbw = d <= 2 ? 1 : d <= 4 ? 2 : 3;
  if (dsize_out) *dsize_out = d;
  if (lbw_out) *lbw_out = lbw;
  if (entry) *entry = ent;
  const double exc_bits = (double)(ns - in_dict) * 32.0;
  return __dadd_rn(__dadd_rn((double)rbw, (double)lbw), __ddiv_rn(exc_bits, (double)ns));
}

// find_best_dictionary over the sorted sample (ns <= NSMAX).
template <typename U, int NSMAX = kRDMaxSamples>
__device__ RDChoice rd_find_best(const U *srt, int ns, int t) {
  constexpr int TB = (int)sizeof(U) * 8;
  double best = 1.7976931348623157e308;
  int best_rbw = 0;
  for (int c = 1; c <= kRDCuts; ++c) {
    const double est = rd_cut<U, NSMAX>(srt, ns, TB - c, t, nullptr, nullptr, nullptr);
    if (est < best) {
      best = est;
      best_rbw = TB - c;
    }
  }
  RDChoice r;
  r.rbw = best_rbw;
  rd_cut<U, NSMAX>(srt, ns, best_rbw, t, &r.dsize, &r.lbw, &r.entry);
  return r;
}

// The dictionary of a choice in every lane's registers, for lookups.
struct RDLookup {
  uint32_t d[kRDDict];
  int dsize, rbw;
  __device__ __forceinline__ RDLookup(const RDChoice &c) : dsize(c.dsize), rbw(c.rbw) {
#pragma unroll
    for (int r = 0; r < kRDDict; ++r) d[r] = __shfl_sync(0xffffffffu, c.entry, r);
  }
  __device__ __forceinline__ RDLookup(const uint16_t *dict, int dsize_, int rbw_)
      : dsize(dsize_), rbw(rbw_) {
#pragma unroll
    for (int r = 0; r < kRDDict; ++r) d[r] = r < dsize_ ? dict[r] : 0u;
  }
  // dictionary index of a left part, dsize when it is not in the dictionary
  __device__ __forceinline__ int index(uint32_t left) const {
    int idx = dsize;
#pragma unroll
    for (int r = kRDDict - 1; r >= 0; --r)
      if (r < dsize && d[r] == left) idx = r;
    return idx;
  }
};

// Exceptions of one vector (left parts not in the dictionary), counted.
template <typename U>
__device__ __forceinline__ int rd_count_exceptions(const U *vec, const RDLookup &lk, int t) {
  int n = 0;
#pragma unroll 4
  for (int k = 0; k < 32; ++k) {
    const uint32_t left = (uint32_t)(vec[32 * k + t] >> lk.rbw);
    n += __popc(__ballot_sync(0xffffffffu, lk.index(left) >= lk.dsize));
  }
  return n;
}

// Writes one vector's ALP-RD encoding:
//   right parts (low rbw bits) FastLanes-packed as U lanes at width rbw at
//     `right` (rbw * 1024 / TB words of U);
//   dictionary indices FastLanes-packed as u16 lanes at width lbw at `left`
//     (lbw * 64 u16 words; thread t writes lanes 2t and 2t + 1 as one
//     32-bit word per line, so `left` must be 4-byte aligned); the index
//     stored at an exception position is dsize masked to lbw bits;
//   exceptions (left part, position) in ascending position at exc / pos.
template <typename U>
__device__ __forceinline__ void rd_write_vector(const U *vec, const RDLookup &lk, int lbw, int t,
                                                U *right, uint16_t *left, uint16_t *exc,
                                                uint16_t *pos) {
  constexpr int TB = (int)sizeof(U) * 8;
  const int rbw = lk.rbw;
  const U rmask = rbw >= TB ? ~(U)0 : (U)(((U)1 << rbw) - 1);
  // right parts, the FastLanes packer's bit writer (base 0)
  if constexpr (TB == 64) {
    const int l = t & 15, h = t >> 4;
    uint32_t *o32 = reinterpret_cast<uint32_t *>(right);
    uint64_t acc = 0;
    int fill = 0, word = 0;
    auto put = [&](uint64_t v, int n) {
      acc |= v << fill;
      fill += n;
      while (fill >= 32) {
        const int j = h * rbw + word++;  // 32-bit word of the lane's stream
        o32[2 * ((size_t)(j >> 1) * 16 + l) + (j & 1)] = (uint32_t)acc;
        acc >>= 32;
        fill -= 32;
      }
    };
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      const uint64_t d = (uint64_t)(vec[l + 16 * (32 * h + k)] & rmask);
      if (rbw <= 32) {
        put(d, rbw);
      } else {
        put(d & 0xFFFFFFFFull, 32);
        put(d >> 32, rbw - 32);
      }
    }
  } else {
    uint64_t acc = 0;
    int fill = 0, word = 0;
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      acc |= (uint64_t)(vec[t + 32 * k] & rmask) << fill;
      fill += rbw;
      while (fill >= 32) {
        right[(size_t)(word++) * 32 + t] = (U)(uint32_t)acc;
        acc >>= 32;
        fill -= 32;
      }
    }
  }
  // dictionary indices: lanes 2t and 2t + 1, 16 values each (lbw <= 3, so a
  // lane's 16 * lbw bits fit one 64-bit accumulator)
  {
    const uint32_t imask = (1u << lbw) - 1u;
    uint64_t a0 = 0, a1 = 0;
#pragma unroll 4
    for (int j = 0; j < 16; ++j) {
      const uint32_t i0 = (uint32_t)lk.index((uint32_t)(vec[2 * t + 64 * j] >> rbw)) & imask;
      const uint32_t i1 = (uint32_t)lk.index((uint32_t)(vec[2 * t + 1 + 64 * j] >> rbw)) & imask;
      a0 |= (uint64_t)i0 << (j * lbw);
      a1 |= (uint64_t)i1 << (j * lbw);
    }
    uint32_t *l32 = reinterpret_cast<uint32_t *>(left);
    for (int i = 0; i < lbw; ++i)
      l32[i * 32 + t] = (uint32_t)((a0 >> (16 * i)) & 0xFFFFu) |
                        ((uint32_t)((a1 >> (16 * i)) & 0xFFFFu) << 16);
  }
  // exceptions in ascending position
  int written = 0;
#pragma unroll 4
  for (int k = 0; k < 32; ++k) {
    const int p = 32 * k + t;
    const uint32_t lp = (uint32_t)(vec[p] >> rbw);
    const bool is_exc = lk.index(lp) >= lk.dsize;
    const unsigned bal = __ballot_sync(0xffffffffu, is_exc);
    if (is_exc) {
      const int slot = written + __popc(bal & ((1u << t) - 1u));
      exc[slot] = (uint16_t)lp;
      pos[slot] = (uint16_t)p;
    }
    written += __popc(bal);
  }
}

// Exclusive scan over NA per-vector size arrays (sizes[a * stride + v], v <
// n) in two launches: k_scan_n_local (offsets within blocks of 1024
// vectors, block totals) and k_scan_n_blocks (offsets of the blocks, column
// totals); the final offset of vector v in array a is offs[a * stride + v] +
// blk[a * bstride + v / 1024].
template <int NA>
__device__ __forceinline__ void block_excl_scan_n(size_t (&x)[NA], size_t (*sw)[32],
                                                  size_t (&tot)[NA]) {
  const int t = threadIdx.x & 31, w = threadIdx.x >> 5;
  size_t inc[NA];
#pragma unroll
  for (int a = 0; a < NA; ++a) inc[a] = x[a];
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      const size_t y = __shfl_up_sync(0xffffffffu, inc[a], o);
      if (t >= o) inc[a] += y;
    }
  }
  if (t == 31) {
#pragma unroll
    for (int a = 0; a < NA; ++a) sw[a][w] = inc[a];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      size_t s = t < (int)(blockDim.x >> 5) ? sw[a][t] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const size_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (t >= o) s += y;
      }
      sw[a][t] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int a = 0; a < NA; ++a) {
    const size_t wo = w ? sw[a][w - 1] : 0;
    tot[a] = sw[a][(blockDim.x >> 5) - 1];
    x[a] = wo + inc[a] - x[a];
  }
}

template <int NA>
__global__ void __launch_bounds__(1024) k_scan_n_local(const uint32_t *sizes, size_t stride,
                                                       size_t n, size_t *offs, size_t *blk,
                                                       size_t bstride) {
  __shared__ size_t sw[NA][32];
  const size_t v = (size_t)blockIdx.x * 1024 + threadIdx.x;
  size_t x[NA], tot[NA];
#pragma unroll
  for (int a = 0; a < NA; ++a) x[a] = v < n ? sizes[a * stride + v] : 0;
  block_excl_scan_n<NA>(x, sw, tot);
#pragma unroll
  for (int a = 0; a < NA; ++a) {
    if (v < n) offs[a * stride + v] = x[a];
    if (threadIdx.x == 0) blk[a * bstride + blockIdx.x] = tot[a];
  }
}

// nb blocks of the local scan; their offsets replace their totals in blk
template <int NA>
__global__ void __launch_bounds__(1024) k_scan_n_blocks(size_t nb, size_t *blk, size_t bstride,
                                                        size_t *totals) {
  __shared__ size_t sw[NA][32];
  size_t carry[NA];
#pragma unroll
  for (int a = 0; a < NA; ++a) carry[a] = 0;
  for (size_t base = 0; base < nb; base += 1024) {
    const size_t i = base + threadIdx.x;
    size_t x[NA], tot[NA];
#pragma unroll
    for (int a = 0; a < NA; ++a) x[a] = i < nb ? blk[a * bstride + i] : 0;
    block_excl_scan_n<NA>(x, sw, tot);
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      if (i < nb) blk[a * bstride + i] = carry[a] + x[a];
      carry[a] += tot[a];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int a = 0; a < NA; ++a) totals[a] = carry[a];
  }
}

}  // namespace flsb200

namespace flsb200 {

// Device workspace of the ALP-RD encoder, sized for cap vectors; the
// encoded column's arrays live here until the next encode.
struct RDWork {
  size_t cap = 0;
  // per rowgroup (at most one per vector): cut and dictionary
  uint8_t *rg_rbw = nullptr, *rg_lbw = nullptr, *rg_dsize = nullptr;
  // per vector
  uint8_t *scheme = nullptr;  // hybrid columns: 0 ALP, 1 ALP-RD
  uint8_t *rbw = nullptr, *lbw = nullptr, *dsize = nullptr;
  uint32_t *dict_idx = nullptr;
  uint16_t *dicts = nullptr;   // 8 per rowgroup (or per vector)
  uint16_t *count = nullptr;
  uint32_t *sizes = nullptr;   // [3][cap]: right words, left u16 words, exceptions
  size_t *offs = nullptr;      // [3][cap]: their exclusive prefixes (final after the pack)
  size_t *blk = nullptr;       // [3][cap / 1024 + 1]
  size_t *totals = nullptr;    // [3]
  // the column
  uint64_t *right = nullptr;   // cap * 1024 words of the value's width (as bytes: cap * 8 KiB)
  uint16_t *left = nullptr;    // cap * 192 u16 (left width <= 3)
  uint16_t *exc = nullptr, *pos = nullptr;  // cap * 1024 each
};

flsgpu_status rd_work_reserve(RDWork &w, size_t n_vecs);
void rd_work_free(RDWork &w);
// Encodes a column as ALP-RD with one dictionary per rowgroup of
// rowgroup_vecs (1..100) vectors; totals[0..2] = right words, left u16
// words, exceptions.
template <typename T>
flsgpu_status run_rd_encode(const T *vals, size_t n_vecs, int rowgroup_vecs, RDWork &w,
                            cudaStream_t s);

}  // namespace flsb200
