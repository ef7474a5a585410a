// batch_query.cu -- fused per-pair query over compressed columns:
//   result[i] = sum of A_i[k] over the positions k with B_i[k] < median(B_i)
// for pairs (A_i: f64 ALP column, B_i: u32 FFOR column of the same length),
// all pairs in one graph of four kernel kinds:
//   * 4 radix-select passes over B (8 bits each, most significant first):
//     each pass histograms the digit of the values that match the prefix
//     chosen so far (k_pq_hist), using each vector's FFOR interval
//     [base, base + 2^w - 1] to skip it or count it whole without decoding
//     where it can, then one warp per pair picks the digit that holds the
//     rank floor((n-1)/2) (k_pq_select);
//   * one pass that adds, per vector, the A values whose B is below the
//     median in the fixed order of the f64 sums (k_pq_sum), one partial per
//     vector, decoding B only for vectors whose interval holds the median
//     and A only for vectors with a selected value;
//   * one block per pair reduces its partials pairwise (k_pq_pairwise).
// The reference has no such query; its multi-column kernel is the model for
// decoding several columns of the same vector in lockstep
// (src/generated-bindings/multi-column-device-kernels.cuh:11-439).
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "../../include/flsgpu_b200_ext.h"

namespace flsb200 {

struct PairEntry {
  ColumnParams a;  // f64 ALP
  ColumnParams b;  // u32 FFOR
};

struct PairState {
  uint32_t prefix;  // digits chosen so far (high bits)
  uint32_t rank;    // rank still to find among the values matching prefix
};

constexpr int kPairChunk = 32;  // vectors per atomic: one per lane of the deciding warp

__device__ __forceinline__ int find_pair(const size_t *prefix, int n, size_t v, int hint) {
  if (hint >= 0 && v >= prefix[hint] && v < prefix[hint + 1]) return hint;
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= v)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void flush_hist(uint32_t *sh, uint32_t *gh, int t) {
  for (int i = t; i < 256; i += 32) {
    const uint32_t c = sh[i];
    if (c) atomicAdd(gh + i, c);
    sh[i] = 0;
  }
}

// Radix-select histogram of pass `pass` (0..3) over every B vector.  A
// vector's values lie in [base, base + 2^w - 1] (when that does not wrap
// past 2^32): if the interval misses the prefix chosen so far the vector is
// skipped, and if it falls in one bin of this pass its valid values are
// counted there without decoding; only the rest are decoded.  A warp takes
// 32 vectors at a time and decides them in parallel, one per lane (one
// round trip for all their metadata), then decodes the undecided ones
// together.
__global__ void __launch_bounds__(256, 2)
    k_pq_hist(const PairEntry *__restrict__ pairs, const size_t *__restrict__ prefix, int n_pairs,
              const PairState *__restrict__ state, uint32_t *hist, int pass,
              unsigned long long *counter, uint32_t *d_status) {
  __shared__ uint32_t s_hist[8][256];
  const int t = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t *sh = s_hist[wib];
  for (int i = t; i < 256; i += 32) sh[i] = 0;
  __syncwarp();
  const size_t total = prefix[n_pairs];
  const int shift = 24 - 8 * pass;
  int cur = -1;  // pair of the shared histogram
  int hint = -1;
  while (true) {
    unsigned long long base = 0;
    if (t == 0) base = atomicAdd(counter, (unsigned long long)kPairChunk);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    // decide, one vector per lane
    const size_t v = base + t;
    int pi = -1, lim = 0, w = 0;
    size_t off = 0;
    uint32_t bbase = 0;
    bool decode = false;
    if (v < total) {
      pi = find_pair(prefix, n_pairs, v, hint);
      const ColumnParams &c = pairs[pi].b;
      const size_t vi = v - prefix[pi];
      const Meta<uint32_t> m = load_meta<uint32_t, K_FFOR>(c, vi);
      const uint32_t *vin;
      XInt<uint32_t> xf;
      if (setup_from_meta<uint32_t, K_FFOR>(c, d_status, m, 0, vin, w, xf)) {
        const size_t rem = c.n_values - vi * VEC;
        lim = rem < (size_t)VEC ? (int)rem : VEC;
        off = m.off;
        bbase = m.base;
        const uint32_t want = pass ? state[pi].prefix >> (shift + 8) : 0u;
        const uint64_t lo = m.base, hi = lo + ((1ull << w) - 1ull);
        decode = true;
        if (hi <= 0xFFFFFFFFull) {
          const uint64_t tlo = lo >> (shift + 8), thi = hi >> (shift + 8);
          const uint32_t dlo = (uint32_t)(lo >> shift) & 255u, dhi = (uint32_t)(hi >> shift) & 255u;
          if (pass > 0 && (thi < want || tlo > want)) {
            decode = false;  // no value matches the prefix
          } else if ((pass == 0 || (tlo == want && thi == want)) && dlo == dhi) {
            decode = false;  // every valid value falls in one bin
            atomicAdd(hist + 256 * (size_t)pi + dlo, (uint32_t)lim);
          }
        }
      }
    }
    hint = __shfl_sync(0xffffffffu, pi, 31);
    if (hint < 0) hint = __shfl_sync(0xffffffffu, pi, 0);
    unsigned todo = __ballot_sync(0xffffffffu, decode);
    while (todo) {
      const int j = __ffs(todo) - 1;
      todo &= todo - 1;
      const int pj = __shfl_sync(0xffffffffu, pi, j);
      const int wj = __shfl_sync(0xffffffffu, w, j);
      const int limj = __shfl_sync(0xffffffffu, lim, j);
      const uint32_t basej = __shfl_sync(0xffffffffu, bbase, j);
      const size_t offj = ((size_t)__shfl_sync(0xffffffffu, (uint32_t)(off >> 32), j) << 32) |
                          __shfl_sync(0xffffffffu, (uint32_t)off, j);
      if (pj != cur) {
        if (cur >= 0) {
          __syncwarp();
          flush_hist(sh, hist + 256 * (size_t)cur, t);
          __syncwarp();
        }
        cur = pj;
      }
      const uint32_t want = pass ? state[pj].prefix >> (shift + 8) : 0u;
      const uint32_t *vin = reinterpret_cast<const uint32_t *>(pairs[pj].b.packed) + offj;
      const XInt<uint32_t> xf{basej};
      decode_values<uint32_t>(vin, wj, t, xf, [&](int idx, uint32_t x, auto...) {
        const bool match = (idx < limj) && (pass == 0 || (x >> (shift + 8)) == want);
        if (match) atomicAdd(&sh[(x >> shift) & 255u], 1u);
      });
    }
  }
  __syncwarp();
  if (cur >= 0) flush_hist(sh, hist + 256 * (size_t)cur, t);
}

// One warp per pair: choose this pass's digit of the rank-th value.
__global__ void k_pq_select(int n_pairs, PairState *state, uint32_t *hist, int pass,
                            uint32_t *d_medians) {
  const int pi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int t = threadIdx.x & 31;
  if (pi >= n_pairs) return;
  uint32_t *h = hist + 256 * (size_t)pi;
  uint32_t c[8], s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    c[i] = h[8 * t + i];
    s += c[i];
  }
  // exclusive scan of the per-lane sums
  uint32_t incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (t >= o) incl += y;
  }
  const uint32_t excl = incl - s;
  const uint32_t rank = state[pi].rank;
  // the lane whose bins contain the rank picks the digit
  int digit = -1;
  uint32_t below = 0;
  if (rank >= excl && rank < incl) {
    uint32_t acc = excl;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (digit < 0 && rank < acc + c[i]) {
        digit = 8 * t + i;
        below = acc;
      }
      acc += c[i];
    }
  }
  const unsigned m = __ballot_sync(0xffffffffu, digit >= 0);
  const int src = m ? __ffs(m) - 1 : 0;
  digit = __shfl_sync(0xffffffffu, digit, src);
  below = __shfl_sync(0xffffffffu, below, src);
#pragma unroll
  for (int i = 0; i < 8; ++i) h[8 * t + i] = 0;
  if (t == 0 && m) {
    const int shift = 24 - 8 * pass;
    state[pi].prefix |= (uint32_t)digit << shift;
    state[pi].rank = rank - below;
    if (pass == 3 && d_medians) d_medians[pi] = state[pi].prefix;
  }
}

// Masked sum.  Per vector, thread t adds A[idx] for idx = t%16 +
// 16*(32*(t/16) + k), k ascending, where B[idx] < median (the order of the
// f64 sums); warp butterfly -> partial.
// B's interval [base, base + 2^w - 1] decides without decoding B when it
// lies wholly below the median (every valid value selected) or at or above
// it (the vector adds nothing and A is not read); otherwise B is decoded
// into one selection bit per value, and the bits a thread needs come from
// the two B lanes that hold its positions (shuffles).  A is decoded into
// the warp's shared memory and patched there before the sum.
__global__ void __launch_bounds__(256, 2)
    k_pq_sum(const PairEntry *__restrict__ pairs, const size_t *__restrict__ prefix, int n_pairs,
             const PairState *__restrict__ state, double *partials, unsigned long long *counter,
             uint32_t *d_status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double *sa = reinterpret_cast<double *>(smem_raw) + wib * VEC;
  const size_t total = prefix[n_pairs];
  const int lane = t & 15, half = t >> 4;
  int hint = -1;
  while (true) {
    unsigned long long base = 0;
    if (t == 0) base = atomicAdd(counter, (unsigned long long)kPairChunk);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    // decide, one vector per lane: 0 nothing selected, 1 all, 2 decode B
    const size_t v = base + t;
    int pi = -1, mode = 0;
    if (v < total) {
      pi = find_pair(prefix, n_pairs, v, hint);
      const PairEntry &pe = pairs[pi];
      const size_t vi = v - prefix[pi];
      const Meta<uint32_t> mb = load_meta<uint32_t, K_FFOR>(pe.b, vi);
      const uint32_t med = state[pi].prefix;
      const uint64_t lo = mb.base, hi = lo + ((1ull << (mb.w <= 32 ? mb.w : 0)) - 1ull);
      mode = 2;
      if (mb.w <= 32 && hi <= 0xFFFFFFFFull) mode = hi < med ? 1 : lo >= med ? 0 : 2;
      if (mode == 0) partials[v] = 0.0;
      else if (mode == 2 && mb.w <= 32) {
        // this lane's straddling vector: its B lines into L2 now
        const char *pb = reinterpret_cast<const char *>(
            reinterpret_cast<const uint32_t *>(pe.b.packed) + mb.off);
        for (int l = 0; l < mb.w; ++l) asm volatile("prefetch.global.L2 [%0];" ::"l"(pb + 128 * l));
      }
    }
    hint = __shfl_sync(0xffffffffu, pi, 31);
    if (hint < 0) hint = __shfl_sync(0xffffffffu, pi, 0);
    unsigned todo = __ballot_sync(0xffffffffu, mode != 0);
    while (todo) {
      const int j = __ffs(todo) - 1;
      todo &= todo - 1;
      const int pj = __shfl_sync(0xffffffffu, pi, j);
      const bool all = __shfl_sync(0xffffffffu, mode, j) == 1;
      const size_t vj = base + j;
      const uint32_t med = state[pj].prefix;
      const size_t vi = vj - prefix[pj];
      const PairEntry &pe = pairs[pj];
      const Meta<double> ma = load_meta<double, K_ALP>(pe.a, vi);
      const Meta<uint32_t> mb = load_meta<uint32_t, K_FFOR>(pe.b, vi);
      double acc = 0.0;
      const uint32_t *bin;
      const uint64_t *ain;
      int wb, wa;
      XInt<uint32_t> xb;
      XAlpF64 xa;
      const bool okb = setup_from_meta<uint32_t, K_FFOR>(pe.b, d_status, mb, t, bin, wb, xb);
      const bool oka = setup_from_meta<double, K_ALP>(pe.a, d_status, ma, t, ain, wa, xa);
      const size_t rem = pe.a.n_values - vi * VEC;
      const int lim = rem < (size_t)VEC ? (int)rem : VEC;
      if (okb && oka) {
        const uint32_t ecnt = pe.a.patch ? ma.ecnt : 0u;
        const double *exc = reinterpret_cast<const double *>(pe.a.exc);
        uint32_t p0 = VEC;
        double e0 = 0.0;
        if ((uint32_t)t < ecnt) {
          p0 = pe.a.pos[ma.eo + t];
          e0 = exc[ma.eo + t];
        }
        uint32_t selA = 0, selB = 0;
        if (!all) {
          prefetch_packed(ain, wa, t);  // A's lines come into L2 while B decodes
          uint32_t bits = 0;
          decode_values<uint32_t>(bin, wb, t, xb, [&](int idx, uint32_t x, auto...) {
            if (idx < lim && x < med) bits |= 1u << (idx >> 5);
          });
          selA = __shfl_sync(0xffffffffu, bits, lane);
          selB = __shfl_sync(0xffffffffu, bits, lane + 16);
        }
        // A into shared memory (a plain store per value keeps this decode's
        // code as small as the single-column kernels'), patched, then summed
        decode_values<double, VAR_DEFAULT | VAR_OCC>(ain, wa, t, xa,
                                                    [&](int idx, double x, auto...) { sa[idx] = x; });
        __syncwarp();
        bool bad = (uint32_t)t < ecnt && p0 >= VEC;
        if (p0 < VEC) sa[p0] = e0;
        bad |= patch_batched<double>(pe.a.pos + ma.eo, exc + ma.eo, 32, ecnt, t,
                                     [&](uint32_t ps, double e) { sa[ps] = e; });
        if (__any_sync(0xffffffffu, bad) && t == 0) flag_status(d_status, FLSGPU_BAD_EXCEPTION);
        __syncwarp();
#pragma unroll 8
        for (int k = 0; k < 32; ++k) {
          const int idx = lane + 16 * (32 * half + k);
          const bool sel = all ? idx < lim
                               : ((((k & 1) ? selB : selA) >> (16 * half + (k >> 1))) & 1u) != 0;
          if (sel) acc = __dadd_rn(acc, sa[idx]);
        }
        __syncwarp();
      }
#pragma unroll
      for (int s = 16; s >= 1; s >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, s));
      if (t == 0) partials[vj] = acc;
    }
  }
}

// One block per pair: pairwise tree (stride doubling) over the pair's
// partials, in aligned chunks of 2048 whose results are combined the same
// way.
__global__ void __launch_bounds__(1024)
    k_pq_pairwise(const size_t *__restrict__ prefix, const double *__restrict__ partials,
                  double *results) {
  __shared__ double s[2048];
  __shared__ double chunks[1024];
  const int pi = blockIdx.x;
  const size_t first = prefix[pi], n = prefix[pi + 1] - prefix[pi];
  const size_t n_chunks = (n + 2047) / 2048;
  for (size_t ch = 0; ch < n_chunks; ++ch) {
    const size_t base = first + ch * 2048;
    const size_t m = n - ch * 2048 < 2048 ? n - ch * 2048 : 2048;
    for (int i = threadIdx.x; i < 2048; i += 1024) s[i] = (size_t)i < m ? partials[base + i] : 0.0;
    __syncthreads();
    for (int st = 1; st < 2048; st <<= 1) {
      const int i = threadIdx.x * 2 * st;
      if (i < 2048 && (size_t)(i + st) < m) s[i] = __dadd_rn(s[i], s[i + st]);
      __syncthreads();
    }
    if (threadIdx.x == 0) chunks[ch] = s[0];
    __syncthreads();
  }
  for (int st = 1; st < (int)n_chunks; st <<= 1) {
    const int i = threadIdx.x * 2 * st;
    if ((size_t)(i + st) < n_chunks) chunks[i] = __dadd_rn(chunks[i], chunks[i + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0) results[pi] = n ? chunks[0] : 0.0;
}

}  // namespace flsb200

struct flsgpu_pair_query {
  int n_pairs = 0;
  flsb200::PairEntry *d_pairs = nullptr;
  size_t *d_prefix = nullptr;
  flsb200::PairState *d_state = nullptr;
  flsb200::PairState *h_state_init = nullptr;
  flsb200::PairState *d_state_init = nullptr;
  uint32_t *d_hist = nullptr;
  double *d_partials = nullptr;
  unsigned long long *d_counter = nullptr;
  double *d_results = nullptr;
  uint32_t *d_medians = nullptr;
  uint32_t *d_status = nullptr;
  size_t total = 0;
  unsigned grid_hist = 0, grid_sum = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace flsb200 {

constexpr size_t kPqSumSmem = 8 * VEC * sizeof(double);
constexpr int kMaxPairVectors = 2048 * 1024;  // chunk results per block (k_pq_pairwise)

static flsgpu_status pq_launch(flsgpu_pair_query *q, cudaStream_t s) {
  flsgpu_status st;
  if ((st = check_cuda(cudaMemcpyAsync(q->d_state, q->d_state_init, sizeof(PairState) * q->n_pairs,
                                       cudaMemcpyDeviceToDevice, s), "reset state")))
    return st;
  if ((st = check_cuda(cudaMemsetAsync(q->d_hist, 0, sizeof(uint32_t) * 256 * q->n_pairs, s), "memset")))
    return st;
  for (int pass = 0; pass < 4; ++pass) {
    if ((st = check_cuda(cudaMemsetAsync(q->d_counter, 0, 8, s), "memset"))) return st;
    k_pq_hist<<<q->grid_hist, 256, 0, s>>>(q->d_pairs, q->d_prefix, q->n_pairs, q->d_state,
                                            q->d_hist, pass, q->d_counter, q->d_status);
    k_pq_select<<<(q->n_pairs * 32 + 255) / 256, 256, 0, s>>>(q->n_pairs, q->d_state, q->d_hist,
                                                              pass, q->d_medians);
    note_launch(2);
  }
  if ((st = check_cuda(cudaMemsetAsync(q->d_counter, 0, 8, s), "memset"))) return st;
  k_pq_sum<<<q->grid_sum, 256, kPqSumSmem, s>>>(q->d_pairs, q->d_prefix, q->n_pairs, q->d_state,
                                                 q->d_partials, q->d_counter, q->d_status);
  k_pq_pairwise<<<q->n_pairs, 1024, 0, s>>>(q->d_prefix, q->d_partials, q->d_results);
  note_launch(2);
  return check_cuda(cudaGetLastError(), "pair query launch");
}

}  // namespace flsb200

using namespace flsb200;

extern "C" {

void flsgpu_pair_query_destroy(flsgpu_pair_query *q);

flsgpu_status flsgpu_pair_query_create(const flsgpu_alp_column *a, const flsgpu_ffor_column *b,
                                       size_t n_pairs, double *d_results, uint32_t *d_medians,
                                       uint32_t *d_status, flsgpu_pair_query **out) {
  if (!out || (n_pairs && (!a || !b || !d_results)))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null pair-query arguments");
  if (n_pairs > (1u << 24)) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "too many pairs");
  std::vector<PairEntry> pe(n_pairs);
  std::vector<size_t> prefix(n_pairs + 1, 0);
  std::vector<PairState> init(n_pairs);
  flsgpu_status s;
  for (size_t i = 0; i < n_pairs; ++i) {
    if ((s = fill(pe[i].a, &a[i], nullptr)) || (s = fill(pe[i].b, &b[i], nullptr))) return s;
    if (a[i].n_values != b[i].n_values)
      return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "pair %zu: A and B differ in length", i);
    if (pe[i].a.n_vecs > (size_t)kMaxPairVectors)
      return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "pair %zu: more than %d vectors", i,
                       kMaxPairVectors);
    prefix[i + 1] = prefix[i] + pe[i].a.n_vecs;
    const size_t n = a[i].n_values;
    init[i] = PairState{0u, n ? (uint32_t)((n - 1) / 2) : 0u};
  }
  auto *q = new flsgpu_pair_query();
  q->n_pairs = (int)n_pairs;
  q->total = prefix[n_pairs];
  q->d_results = d_results;
  q->d_medians = d_medians;
  q->d_status = d_status;
  const size_t np = n_pairs ? n_pairs : 1;
  if ((s = check_cuda(cudaMalloc(&q->d_pairs, sizeof(PairEntry) * np), "cudaMalloc")) ||
      (s = check_cuda(cudaMalloc(&q->d_prefix, sizeof(size_t) * (n_pairs + 1)), "cudaMalloc")) ||
      (s = check_cuda(cudaMalloc(&q->d_state, sizeof(PairState) * np), "cudaMalloc")) ||
      (s = check_cuda(cudaMalloc(&q->d_state_init, sizeof(PairState) * np), "cudaMalloc")) ||
      (s = check_cuda(cudaMalloc(&q->d_hist, sizeof(uint32_t) * 256 * np), "cudaMalloc")) ||
      (s = check_cuda(cudaMalloc(&q->d_partials, sizeof(double) * (q->total ? q->total : 1)), "cudaMalloc")) ||
      (s = check_cuda(cudaMalloc(&q->d_counter, 8), "cudaMalloc"))) {
    flsgpu_pair_query_destroy(q);
    return s;
  }
  if (n_pairs) {
    s = check_cuda(cudaMemcpy(q->d_pairs, pe.data(), sizeof(PairEntry) * n_pairs, cudaMemcpyHostToDevice), "copy");
    if (!s) s = check_cuda(cudaMemcpy(q->d_state_init, init.data(), sizeof(PairState) * n_pairs, cudaMemcpyHostToDevice), "copy");
  }
  if (!s) s = check_cuda(cudaMemcpy(q->d_prefix, prefix.data(), sizeof(size_t) * (n_pairs + 1), cudaMemcpyHostToDevice), "copy");
  if (s) {
    flsgpu_pair_query_destroy(q);
    return s;
  }
  static int bps_hist = 0, bps_sum = 0;
  if (!bps_hist) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps_hist, k_pq_hist, 256, 0);
    cudaFuncSetAttribute(k_pq_sum, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPqSumSmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps_sum, k_pq_sum, 256, kPqSumSmem);
    if (bps_hist < 1) bps_hist = 1;
    if (bps_sum < 1) bps_sum = 1;
  }
  q->grid_hist = persistent_blocks(q->total ? q->total : 1, 8, bps_hist);
  q->grid_sum = persistent_blocks(q->total ? q->total : 1, 8, bps_sum);
  *out = q;
  return FLSGPU_OK;
}

flsgpu_status flsgpu_pair_query_run(flsgpu_pair_query *q, flsgpu_stream stream) {
  if (!q) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null query");
  if (q->n_pairs == 0) return FLSGPU_OK;
  return pq_launch(q, (cudaStream_t)stream);
}

flsgpu_status flsgpu_pair_query_capture_graph(flsgpu_pair_query *q, flsgpu_stream stream) {
  if (!q) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null query");
  cudaStream_t s = (cudaStream_t)stream;
  bool own = false;
  flsgpu_status st;
  if (!s) {
    if ((st = check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream"))) return st;
    own = true;
  }
  if (q->exec) cudaGraphExecDestroy(q->exec);
  if (q->graph) cudaGraphDestroy(q->graph);
  q->exec = nullptr;
  q->graph = nullptr;
  st = check_cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture");
  if (!st) {
    flsgpu_status ls = q->n_pairs ? pq_launch(q, s) : FLSGPU_OK;
    flsgpu_status es = check_cuda(cudaStreamEndCapture(s, &q->graph), "end capture");
    st = ls ? ls : es;
  }
  if (!st) st = check_cuda(cudaGraphInstantiate(&q->exec, q->graph, 0), "instantiate");
  if (own) cudaStreamDestroy(s);
  return st;
}

flsgpu_status flsgpu_pair_query_replay(flsgpu_pair_query *q, flsgpu_stream stream) {
  if (!q || !q->exec) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "no captured graph");
  flsgpu_status st = check_cuda(cudaGraphLaunch(q->exec, (cudaStream_t)stream), "graph launch");
  if (!st) note_launch();
  return st;
}

void flsgpu_pair_query_destroy(flsgpu_pair_query *q) {
  if (!q) return;
  if (q->exec) cudaGraphExecDestroy(q->exec);
  if (q->graph) cudaGraphDestroy(q->graph);
  cudaFree(q->d_pairs);
  cudaFree(q->d_prefix);
  cudaFree(q->d_state);
  cudaFree(q->d_state_init);
  cudaFree(q->d_hist);
  cudaFree(q->d_partials);
  cudaFree(q->d_counter);
  delete q;
}

}  // extern "C"
