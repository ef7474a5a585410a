// batch.cuh -- the persistent batched decode kernel, one instantiation per
// value type (batch_{u32,u64,f32,f64}.cu), so that each type gets the
// register allocation (and occupancy) of its own widest unpacker instead of
// the maximum over all types.
#pragma once

#include "kernels.cuh"

namespace flsb200 {

struct BatchEntry {
  KernelParams p;       // one column and its output
  uint32_t kind;        // K_BP, K_FFOR, K_ALP, K_ALPX
  uint32_t pad;
};

constexpr int kBatchChunk = 32;  // vectors taken per atomic

// Column of global vector v: prefix has n_cols + 1 entries, prefix[0] = 0;
// the hint (last column) is checked first.
__device__ __forceinline__ int find_column(const size_t *prefix, int n_cols, size_t v, int hint) {
  if (hint >= 0 && v >= prefix[hint] && v < prefix[hint + 1]) return hint;
  if (hint >= 0 && hint + 1 < n_cols && v >= prefix[hint + 1] && v < prefix[hint + 2])
    return hint + 1;
  int lo = 0, hi = n_cols;  // invariant: prefix[lo] <= v < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= v)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// f64 ALP decodes faster register-capped at two blocks per SM (wide widths
// in two runs of 16 values), as the single-column autotuning found; u64
// FFOR keeps the register-rich kernel.
template <typename T> constexpr int batch_var() {
  return std::is_same<T, double>::value ? (VAR_DEFAULT | VAR_OCC) : VAR_DEFAULT;
}
template <typename T> constexpr int batch_min_blocks() { return min_blocks<T, batch_var<T>()>(); }

// Persistent decode of every vector of a group of columns of one value
// type.  Warps take chunks of kBatchChunk vectors of the group's index space
// from an atomic counter; the column descriptor is staged in shared memory
// when a warp moves to another column; the next vector's metadata is loaded
// before the current one is decoded when both are in the same column.
// XK: the group's float column kind (K_ALP or K_ALPX; one kernel each so
// that neither carries the other's registers); integer groups mix BP and
// FFOR columns (XK = K_FFOR).
template <typename T, int XK>
__global__ void __launch_bounds__(256, batch_min_blocks<T>())
    k_batch(const BatchEntry *__restrict__ table, const size_t *__restrict__ prefix, int n_cols,
            unsigned long long *counter) {
  constexpr bool FLOAT = std::is_floating_point<T>::value;
  const int t = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const size_t total = prefix[n_cols];
  __shared__ KernelParams s_p[8];
  __shared__ uint32_t s_kind[8];
  int col = -1;
  while (true) {
    unsigned long long base = 0;
    if (t == 0) base = atomicAdd(counter, (unsigned long long)kBatchChunk);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    const size_t end = base + kBatchChunk < total ? base + kBatchChunk : total;
    Meta<T> meta;
    bool have_meta = false;
    for (size_t v = base; v < end; ++v) {
      const int c = find_column(prefix, n_cols, v, col);
      if (c != col) {
        __syncwarp();
        const uint32_t *src = reinterpret_cast<const uint32_t *>(&table[c].p);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&s_p[wib]);
        for (int i = t; i < (int)(sizeof(KernelParams) / 4); i += 32) dst[i] = src[i];
        if (t == 0) s_kind[wib] = table[c].kind;
        __syncwarp();
        col = c;
        have_meta = false;
      }
      const KernelParams &p = s_p[wib];
      const uint32_t kind = s_kind[wib];
      const size_t vi = v - prefix[c];
      if constexpr (FLOAT) {
        (void)kind;
        const Meta<T> cur = have_meta ? meta : load_meta<T, XK>(p.c, vi, t);
        have_meta = v + 1 < end && v + 1 < prefix[c + 1];
        if (have_meta) meta = load_meta<T, XK>(p.c, vi + 1, t);
        store_one<T, XK, batch_var<T>()>(p, vi, cur, t);
      } else {
        const Meta<T> cur = have_meta ? meta
                            : (kind == K_BP ? load_meta<T, K_BP>(p.c, vi)
                                            : load_meta<T, K_FFOR>(p.c, vi));
        have_meta = v + 1 < end && v + 1 < prefix[c + 1];
        if (have_meta)
          meta = kind == K_BP ? load_meta<T, K_BP>(p.c, vi + 1) : load_meta<T, K_FFOR>(p.c, vi + 1);
        if (kind == K_BP)
          store_one<T, K_BP, VAR_DEFAULT>(p, vi, cur, t);
        else
          store_one<T, K_FFOR, VAR_DEFAULT>(p, vi, cur, t);
      }
    }
  }
}

template <typename T, int XK> struct BatchLauncher {
  static int blocks_per_sm() {
    static int bps = 0;
    if (bps == 0) {
      int b = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch<T, XK>, 256, 0);
      bps = b > 0 ? b : 1;
    }
    return bps;
  }
  static flsgpu_status launch(const BatchEntry *table, const size_t *prefix, int n_cols,
                              size_t total_vecs, unsigned long long *counter, cudaStream_t s) {
    flsgpu_status st =
        check_cuda(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s), "memset");
    if (st) return st;
    const unsigned grid = persistent_blocks(total_vecs ? total_vecs : 1, 8, blocks_per_sm());
    k_batch<T, XK><<<grid, 256, 0, s>>>(table, prefix, n_cols, counter);
    note_launch();
    return check_cuda(cudaGetLastError(), "k_batch launch");
  }
};

// Launches k_batch over one group (defined in batch_{u32,u64,f32,f64}.cu);
// alpx selects the ALP-extended kernel of the float types.
flsgpu_status launch_batch_u32(const BatchEntry *, const size_t *, int, size_t,
                               unsigned long long *, cudaStream_t, int alpx);
flsgpu_status launch_batch_u64(const BatchEntry *, const size_t *, int, size_t,
                               unsigned long long *, cudaStream_t, int alpx);
flsgpu_status launch_batch_f32(const BatchEntry *, const size_t *, int, size_t,
                               unsigned long long *, cudaStream_t, int alpx);
flsgpu_status launch_batch_f64(const BatchEntry *, const size_t *, int, size_t,
                               unsigned long long *, cudaStream_t, int alpx);

}  // namespace flsb200
