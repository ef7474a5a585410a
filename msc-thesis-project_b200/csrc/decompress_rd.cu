// decompress_rd.cu -- ALP-RD decoding (the reference has CPU code only:
// rd_encoder::decode, src/alp/rd.hpp:146-172).
//
// Per vector, one warp; all of the vector's loads are issued first (the
// left index words, the dictionary, the first 32 exceptions, the right
// parts, which an L2 prefetch one vector earlier has brought close):
//   1. unpack the right parts (u64 half-lanes / u32 lanes, FFOR base 0) into
//      shared memory;
//   2. unpack the u16 FastLanes left-index lanes (thread t holds lanes 2t
//      and 2t+1 in one 32-bit word per line), look each index up in the
//      vector's 8-entry dictionary (held one entry per lane, fetched with a
//      shuffle) and stage the 1024 left parts in shared memory;
//   3. overwrite the left parts of the exception positions (warp-parallel:
//      positions of a vector are distinct);
//   4. write (left << right_bw) | right as the output bit pattern, 32
//      consecutive values per warp store.
#include <cstring>

#include "rd_decode.cuh"

namespace flsb200 {

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 2 : 1) k_alprd(const RDParams p) {
  using U = typename UintOf<T>::U;
  constexpr int MAXW = sizeof(U) * 8;
  extern __shared__ __align__(16) unsigned char rd_smem[];
  // per warp: the right parts (1024 U) and the left parts (1024 u16)
  U *sr = reinterpret_cast<U *>(rd_smem) + (threadIdx.x >> 5) * VEC;
  uint16_t *sl = reinterpret_cast<uint16_t *>(rd_smem + 8 * VEC * sizeof(U)) + (threadIdx.x >> 5) * VEC;
  const int t = threadIdx.x & 31;
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const U *right_all = reinterpret_cast<const U *>(p.right_packed);

  RDMeta m0{}, m1{};
  if (gw < p.n_vecs) {
    m0 = rd_meta(p, gw);
    if (m0.rbw <= MAXW) prefetch_packed(right_all + m0.roff, m0.rbw, t);
  }
  if (gw + nw < p.n_vecs) m1 = rd_meta(p, gw + nw);
  for (size_t vi = gw; vi < p.n_vecs; vi += nw) {
    const RDMeta m = m0;
    // the next vector's right part is fetched into L2 while this one is
    // decoded; metadata of the vector after it is in flight
    if (vi + nw < p.n_vecs && m1.rbw <= MAXW) prefetch_packed(right_all + m1.roff, m1.rbw, t);
    m0 = m1;
    if (vi + 2 * nw < p.n_vecs) m1 = rd_meta(p, vi + 2 * nw);
    if (m.rbw > MAXW || m.lbw > 16) {
      if (t == 0 && p.d_status) atomicOr(p.d_status, FLSGPU_BAD_BIT_WIDTH);
      continue;
    }
    rd_decode_vector<T>(p, vi, m, t, sr, sl);
    __syncwarp();
  }
}

template <typename T>
static flsgpu_status decompress_rd(const flsgpu_alprd_column *c, T *d_out,
                                   const flsgpu_decode_opts *o, flsgpu_stream stream) {
  flsgpu_status s = check_opts(o);
  if (s) return s;
  RDParams p{};
  if ((s = fill_rd(p, c))) return s;
  if (p.n_vecs == 0) return FLSGPU_OK;
  if (!d_out) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null output");
  if (((uintptr_t)d_out % sizeof(T)) != 0)
    return set_error(FLSGPU_ERR_MISALIGNED, "output not aligned");
  p.d_status = o ? o->d_status : nullptr;
  p.out = d_out;
  constexpr size_t smem = 8 * VEC * (sizeof(T) + sizeof(uint16_t));
  static int bps = 0;
  if (bps == 0) {
    cudaFuncSetAttribute(k_alprd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_alprd<T>, 256, smem);
    bps = b > 0 ? b : 1;
  }
  const unsigned grid = persistent_blocks(p.n_vecs, 8, bps);
  k_alprd<T><<<grid, 256, smem, (cudaStream_t)stream>>>(p);
  note_launch();
  return check_cuda(cudaGetLastError(), "k_alprd launch");
}

}  // namespace flsb200

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_decompress_alprd_f32(const flsgpu_alprd_column *c, float *o,
                                          const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress_rd<float>(c, o, op, s);
}

flsgpu_status flsgpu_decompress_alprd_f64(const flsgpu_alprd_column *c, double *o,
                                          const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress_rd<double>(c, o, op, s);
}

}  // extern "C"
