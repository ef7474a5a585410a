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

#include "kernels.cuh"

namespace flsb200 {

struct RDParams {
  size_t n_values, n_vecs;
  const void *right_packed;
  const uint8_t *right_bw;
  const size_t *right_offs;
  const uint16_t *left_packed;
  const uint8_t *left_bw;
  const size_t *left_offs;
  const uint16_t *dicts;
  const uint32_t *dict_index;
  const size_t *exc_offs;
  const uint16_t *exc;
  const uint16_t *pos;
  const uint16_t *counts;
  uint32_t *d_status;
  void *out;
};

// Per-vector metadata, loaded two vectors ahead of its use.
struct RDMeta {
  size_t loff, roff, eo;
  uint32_t di, cnt;
  int rbw, lbw;
};

__device__ __forceinline__ RDMeta rd_meta(const RDParams &p, size_t vi) {
  RDMeta m;
  m.rbw = p.right_bw[vi];
  m.lbw = p.left_bw[vi];
  m.di = p.dict_index[vi];
  m.loff = p.left_offs[vi];
  m.roff = p.right_offs[vi];
  m.cnt = p.counts[vi];
  m.eo = p.exc_offs[vi];
  return m;
}

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
  U *out_all = reinterpret_cast<U *>(p.out);
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
    // every load of the vector is issued before any is used: the left
    // index words, the dictionary entry, the first 32 exceptions, then the
    // right parts (decoded into shared memory as they arrive)
    uint32_t lw[16];
    const uint32_t *lin = reinterpret_cast<const uint32_t *>(p.left_packed + m.loff);
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (j < m.lbw) lw[j] = ld_stream_u32(lin + j * 32 + t);
    const uint16_t dct = (t < 8) ? p.dicts[8 * (size_t)m.di + t] : 0;
    uint32_t p0 = VEC;
    uint16_t e0 = 0;
    if ((uint32_t)t < m.cnt) {
      p0 = p.pos[m.eo + t];
      e0 = p.exc[m.eo + t];
    }
    const XInt<U> ident{0};
    decode_values<U, VAR_DEFAULT | VAR_OCC>(right_all + m.roff, m.rbw, t, ident,
                     [&](int idx, U r, auto...) { sr[idx] = r; });
    switch_width16(m.lbw, [&](auto wc) {
      constexpr int W = decltype(wc)::value;
      unpack_pair16<W>(lw, [&](int sub, int k, uint32_t idx) {
        // indices >= 8 only occur at exception positions (patched below)
        const uint16_t left = (uint16_t)__shfl_sync(0xffffffffu, (uint32_t)dct, idx < 8 ? idx : 7);
        sl[(2 * t + sub) + 64 * k] = left;
      });
    });
    __syncwarp();
    bool bad = (uint32_t)t < m.cnt && p0 >= VEC;
    if (p0 < VEC) sl[p0] = e0;
    for (uint32_t i = t + 32; i < m.cnt; i += 32) {
      const uint32_t ps = p.pos[m.eo + i];
      if (ps < VEC)
        sl[ps] = p.exc[m.eo + i];
      else
        bad = true;
    }
    if (__any_sync(0xffffffffu, bad) && t == 0 && p.d_status)
      atomicOr(p.d_status, FLSGPU_BAD_EXCEPTION);
    __syncwarp();
    const size_t vbase = vi * VEC;
    const size_t rem = p.n_values - vbase;
    const int lim = rem < (size_t)VEC ? (int)rem : VEC;
    U *out = out_all + vbase;
    const int rbw = m.rbw;
#pragma unroll 8
    for (int i = 0; i < VEC / 32; ++i) {
      const int idx = t + 32 * i;
      const U l = rbw >= MAXW ? U(0) : (U)((U)sl[idx] << rbw);
      if (idx < lim) out[idx] = l | sr[idx];
    }
    __syncwarp();
  }
}

template <typename T>
static flsgpu_status decompress_rd(const flsgpu_alprd_column *c, T *d_out,
                                   const flsgpu_decode_opts *o, flsgpu_stream stream) {
  flsgpu_status s = check_opts(o);
  if (s) return s;
  if (!c) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  RDParams p{};
  p.n_values = c->n_values;
  p.n_vecs = vecs_of(c->n_values);
  if (p.n_vecs == 0) return FLSGPU_OK;
  if (!d_out) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null output");
  if (((uintptr_t)d_out % sizeof(T)) != 0)
    return set_error(FLSGPU_ERR_MISALIGNED, "output not aligned");
  if (((uintptr_t)c->left.packed_array % 4) != 0)
    return set_error(FLSGPU_ERR_MISALIGNED, "left parts must be 4-byte aligned");
  p.right_packed = c->right.packed_array;
  p.right_bw = c->right.bit_widths;
  p.right_offs = c->right.vector_offsets;
  p.left_packed = reinterpret_cast<const uint16_t *>(c->left.packed_array);
  p.left_bw = c->left.bit_widths;
  p.left_offs = c->left.vector_offsets;
  p.dicts = c->dictionaries;
  p.dict_index = c->dictionary_indices;
  p.exc_offs = c->exceptions_offsets;
  p.exc = c->exceptions;
  p.pos = c->positions;
  p.counts = c->counts;
  if (!p.right_bw || !p.right_offs || !p.left_bw || !p.left_offs || !p.dicts || !p.dict_index ||
      !p.counts || !p.exc_offs)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null ALP-RD array");
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
