// rd_encode.cu -- the GPU ALP-RD column encoder (rd_encoder::init + encode,
// src/alp/rd.hpp:28-140, per rowgroup as upstream ALP samples it; the
// device code is in rd_encode.cuh).  Four launches:
//   k_rd_init   one warp per rowgroup: first-level sample (every 12th
//               vector of the rowgroup, 32 values at stride 32 of each,
//               sampler.hpp:11-48), sort, cut search, dictionary;
//   k_rd_count  one warp per vector: exception count and packed sizes;
//   scan        offsets of the right parts, left indices and exceptions;
//   k_rd_pack   one warp per vector: packed right parts, packed left
//               indices, exceptions, all at their final offsets.
#include "rd_encode.cuh"

namespace flsb200 {

template <typename T>
__global__ void __launch_bounds__(128) k_rd_init(const T *__restrict__ vals, size_t n_vecs,
                                                 int rg_vecs, RDWork w) {
  using U = typename RDT<T>::U;
  __shared__ U s_smp[4][kRDMaxSamples], s_srt[4][kRDMaxSamples];
  const int t = threadIdx.x & 31, wib = threadIdx.x >> 5;
  U *smp = s_smp[wib], *srt = s_srt[wib];
  const U *u = reinterpret_cast<const U *>(vals);
  const size_t n_rg = (n_vecs + rg_vecs - 1) / rg_vecs;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t r = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n_rg; r += nw) {
    const size_t v0 = r * (size_t)rg_vecs;
    const int nv = (int)(n_vecs - v0 < (size_t)rg_vecs ? n_vecs - v0 : (size_t)rg_vecs);
    int ns = 0;
    __syncwarp();
    for (int s = 0; s < nv; s += 12) {  // ROWGROUP_SAMPLES_JUMP = 12
      smp[ns + t] = u[(v0 + s) * VEC + 32 * t];
      ns += 32;
    }
    __syncwarp();
    rd_rank_sort<U>(smp, ns, srt, t);
    const RDChoice c = rd_find_best<U>(srt, ns, t);
    if (t < kRDDict) w.dicts[r * kRDDict + t] = (uint16_t)(t < c.dsize ? c.entry : 0u);
    if (t == 0) {
      w.rg_rbw[r] = (uint8_t)c.rbw;
      w.rg_lbw[r] = (uint8_t)c.lbw;
      w.rg_dsize[r] = (uint8_t)c.dsize;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_rd_count(const T *__restrict__ vals, size_t n_vecs,
                                                  int rg_vecs, RDWork w) {
  using U = typename RDT<T>::U;
  constexpr int NL = VEC / RDT<T>::TB;
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const size_t r = v / (size_t)rg_vecs;
    const int rbw = w.rg_rbw[r], lbw = w.rg_lbw[r], dsize = w.rg_dsize[r];
    const RDLookup lk(w.dicts + r * kRDDict, dsize, rbw);
    const int n_exc = rd_count_exceptions<U>(reinterpret_cast<const U *>(vals) + v * VEC, lk, t);
    if (t == 0) {
      w.rbw[v] = (uint8_t)rbw;
      w.lbw[v] = (uint8_t)lbw;
      w.dsize[v] = (uint8_t)dsize;
      w.dict_idx[v] = (uint32_t)r;
      w.count[v] = (uint16_t)n_exc;
      w.sizes[v] = (uint32_t)(rbw * NL);
      w.sizes[w.cap + v] = (uint32_t)(lbw * 64);
      w.sizes[2 * w.cap + v] = (uint32_t)n_exc;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_rd_pack(const T *__restrict__ vals, size_t n_vecs,
                                                 RDWork w) {
  using U = typename RDT<T>::U;
  const int t = threadIdx.x & 31;
  const size_t nb = (w.cap + 1023) / 1024;  // the block offsets' stride
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const size_t orr = w.offs[v] + w.blk[v >> 10];
    const size_t ol = w.offs[w.cap + v] + w.blk[nb + (v >> 10)];
    const size_t oe = w.offs[2 * w.cap + v] + w.blk[2 * nb + (v >> 10)];
    const uint32_t di = w.dict_idx[v];
    const RDLookup lk(w.dicts + (size_t)di * kRDDict, w.dsize[v], w.rbw[v]);
    rd_write_vector<U>(reinterpret_cast<const U *>(vals) + v * VEC, lk, w.lbw[v], t,
                       reinterpret_cast<U *>(w.right) + orr, w.left + ol, w.exc + oe, w.pos + oe);
    __syncwarp();
    if (t == 0) {
      w.offs[v] = orr;
      w.offs[w.cap + v] = ol;
      w.offs[2 * w.cap + v] = oe;
    }
  }
}

template <typename T> static unsigned rd_grid(size_t n) {
  return persistent_blocks(n ? n : 1, 8, 4);
}

template <typename T>
flsgpu_status run_rd_encode(const T *vals, size_t n_vecs, int rg_vecs, RDWork &w,
                            cudaStream_t s) {
  if (!n_vecs) return FLSGPU_OK;
  if (rg_vecs < 1 || rg_vecs > 100)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "ALP-RD rowgroup of %d vectors (1..100)", rg_vecs);
  if (n_vecs > w.cap) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "ALP-RD workspace too small");
  const size_t n_rg = (n_vecs + rg_vecs - 1) / rg_vecs;
  k_rd_init<T><<<persistent_blocks(n_rg, 4, 8), 128, 0, s>>>(vals, n_vecs, rg_vecs, w);
  k_rd_count<T><<<rd_grid<T>(n_vecs), 256, 0, s>>>(vals, n_vecs, rg_vecs, w);
  const size_t nb = (n_vecs + 1023) / 1024, bstride = (w.cap + 1023) / 1024;
  k_scan_n_local<3><<<(unsigned)nb, 1024, 0, s>>>(w.sizes, w.cap, n_vecs, w.offs, w.blk, bstride);
  k_scan_n_blocks<3><<<1, 1024, 0, s>>>(nb, w.blk, bstride, w.totals);
  k_rd_pack<T><<<rd_grid<T>(n_vecs), 256, 0, s>>>(vals, n_vecs, w);
  note_launch(5);
  return check_cuda(cudaGetLastError(), "ALP-RD encode");
}

template flsgpu_status run_rd_encode<double>(const double *, size_t, int, RDWork &, cudaStream_t);
template flsgpu_status run_rd_encode<float>(const float *, size_t, int, RDWork &, cudaStream_t);

template <typename P> static P *rd_alloc(size_t n, flsgpu_status &st) {
  void *p = nullptr;
  if (st == FLSGPU_OK) st = check_cuda(cudaMalloc(&p, (n ? n : 1) * sizeof(P) + 16), "cudaMalloc");
  return static_cast<P *>(p);
}

void rd_work_free(RDWork &w) {
  for (void *p : {(void *)w.rg_rbw, (void *)w.rg_lbw, (void *)w.rg_dsize, (void *)w.scheme,
                  (void *)w.rbw, (void *)w.lbw, (void *)w.dsize, (void *)w.dict_idx,
                  (void *)w.dicts, (void *)w.count, (void *)w.sizes, (void *)w.offs, (void *)w.blk,
                  (void *)w.totals, (void *)w.right, (void *)w.left, (void *)w.exc, (void *)w.pos})
    if (p) cudaFree(p);
  w = RDWork{};
}

flsgpu_status rd_work_reserve(RDWork &w, size_t n_vecs) {
  if (n_vecs <= w.cap) return FLSGPU_OK;
  rd_work_free(w);
  flsgpu_status st = FLSGPU_OK;
  const size_t n = n_vecs, nb = (n + 1023) / 1024;
  w.rg_rbw = rd_alloc<uint8_t>(n, st);
  w.rg_lbw = rd_alloc<uint8_t>(n, st);
  w.rg_dsize = rd_alloc<uint8_t>(n, st);
  w.scheme = rd_alloc<uint8_t>(n, st);
  w.rbw = rd_alloc<uint8_t>(n, st);
  w.lbw = rd_alloc<uint8_t>(n, st);
  w.dsize = rd_alloc<uint8_t>(n, st);
  w.dict_idx = rd_alloc<uint32_t>(n, st);
  w.dicts = rd_alloc<uint16_t>(n * kRDDict, st);
  w.count = rd_alloc<uint16_t>(n, st);
  w.sizes = rd_alloc<uint32_t>(3 * n, st);
  w.offs = rd_alloc<size_t>(3 * n, st);
  w.blk = rd_alloc<size_t>(3 * nb, st);
  w.totals = rd_alloc<size_t>(4, st);
  w.right = rd_alloc<uint64_t>(n * VEC, st);
  w.left = rd_alloc<uint16_t>(n * 192, st);
  w.exc = rd_alloc<uint16_t>(n * VEC, st);
  w.pos = rd_alloc<uint16_t>(n * VEC, st);
  if (st == FLSGPU_OK)
    w.cap = n;
  else
    rd_work_free(w);
  return st;
}

}  // namespace flsb200
