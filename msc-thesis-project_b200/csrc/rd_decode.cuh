// rd_decode.cuh -- ALP-RD decoding of one vector by one warp (the
// reference has CPU code only: rd_encoder::decode, src/alp/rd.hpp:146-172),
// shared by the ALP-RD column kernel (decompress_rd.cu) and the hybrid
// ALP / ALP-RD column kernel (decompress_hybrid.cu).
//
// All of the vector's loads are issued first (the left index words, the
// dictionary, the first 32 exceptions, the right parts, which an L2
// prefetch one vector earlier has brought close):
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
#pragma once

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

// The kernel parameters of an ALP-RD column descriptor (host side).
static inline flsgpu_status fill_rd(RDParams &p, const flsgpu_alprd_column *c) {
  if (!c) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  p.n_values = c->n_values;
  p.n_vecs = vecs_of(c->n_values);
  if (p.n_vecs == 0) return FLSGPU_OK;
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
  return FLSGPU_OK;
}

// Decodes vector vi (metadata m) into p.out; sr / sl: the warp's shared
// staging of the right parts (1024 U) and left parts (1024 u16).
template <typename T>
__device__ __forceinline__ void rd_decode_vector(const RDParams &p, size_t vi, const RDMeta &m,
                                                 int t, typename UintOf<T>::U *sr, uint16_t *sl) {
  using U = typename UintOf<T>::U;
  constexpr int MAXW = sizeof(U) * 8;
  U *out_all = reinterpret_cast<U *>(p.out);
  const U *right_all = reinterpret_cast<const U *>(p.right_packed);
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
    bad |= patch_batched<uint16_t>(p.pos + m.eo, p.exc + m.eo, 32, m.cnt, t,
                                   [&](uint32_t ps, uint16_t e) { sl[ps] = e; });
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
}

}  // namespace flsb200
