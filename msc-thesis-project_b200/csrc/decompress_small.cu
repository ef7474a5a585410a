// decompress_small.cu -- BP / FFOR decoding of 8- and 16-bit FastLanes
// columns (fls::unpack / fls::unffor for uint8_t and uint16_t,
// src/fls/fls-bindings.hpp:8-52; the reference decodes these widths on the
// CPU only).
//
// Layout as for the wider types: a vector is 1024 values in N lanes (128 for
// u8, 64 for u16) of 1024 / N values; value k of lane l is element l + k N;
// stream word j of lane l is packed[j N + l]; a vector packed at width w
// occupies w N words (w * 128 bytes).  One warp per vector over a
// persistent grid: thread t reads the 32-bit words j * 32 + t, which hold
// line j of its S = 32 / E lanes (E = 8 or 16 bits per lane word), unpacks
// the S lanes' values and writes, for each k, its S adjacent outputs (lanes
// S t .. S t + S - 1 of row k) as one 32-bit store, so a warp store covers
// 128 contiguous bytes.
#include "kernels.cuh"

namespace flsb200 {

template <int E> struct SmallLanes {
  static constexpr int S = 32 / E;        // lanes per thread
  static constexpr int NL = 1024 / E;     // lanes per vector
  static constexpr int VPL = E;           // values per lane
  static constexpr uint32_t EMASK = (1u << E) - 1u;
};

// Value k of sub-lane `sub` from the thread's words w[j] (line j).
template <int E, int W>
__device__ __forceinline__ uint32_t small_value(const uint32_t *w, int sub, int k) {
  if (W == 0) return 0u;
  constexpr uint32_t EM = SmallLanes<E>::EMASK;
  const int bit = k * W, j = bit / E, o = bit % E;
  uint32_t v = ((w[j] >> (E * sub)) & EM) >> o;
  if (o + W > E) v |= ((w[j + 1] >> (E * sub)) & EM) << (E - o);
  return v & ((1u << W) - 1u);
}

struct SmallParams {
  size_t n_values, n_vecs;
  const uint32_t *packed;   // as 32-bit words
  const uint8_t *bw;
  const size_t *offs;       // in lane words (E bits)
  const void *bases;        // E-bit per vector, or null (BP)
  uint32_t *d_status;
  void *out;
  size_t n_packed;          // bound in lane words (0: none)
};

template <int E>
__global__ void __launch_bounds__(256) k_store_small(const SmallParams p) {
  using L = SmallLanes<E>;
  using UT = typename std::conditional<E == 8, uint8_t, uint16_t>::type;
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  UT *out_all = reinterpret_cast<UT *>(p.out);
  for (size_t vi = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; vi < p.n_vecs; vi += nw) {
    const int w = p.bw[vi];
    const size_t off = p.offs[vi];
    const uint32_t base = p.bases ? (uint32_t)reinterpret_cast<const UT *>(p.bases)[vi] : 0u;
    uint32_t bad = 0;
    if (w > E) bad |= FLSGPU_BAD_BIT_WIDTH;
    if (p.n_packed && (off > p.n_packed || (size_t)w * L::NL > p.n_packed - off)) bad |= FLSGPU_BAD_OFFSET;
    // a vector's packed words start on a 32-bit boundary: offsets are whole
    // multiples of N lane words (w N E bits = w * 128 bytes per vector)
    if ((off * E) % 32) bad |= FLSGPU_BAD_OFFSET;
    if (bad) {
      if (t == 0) flag_status(p.d_status, bad);
      continue;
    }
    const uint32_t *vin = p.packed + off * E / 32;
    const size_t vbase = vi * VEC;
    const size_t rem = p.n_values - vbase;
    const int lim = rem < (size_t)VEC ? (int)rem : VEC;
    UT *out = out_all + vbase;
    uint32_t *out32 = reinterpret_cast<uint32_t *>(out);
    auto emit = [&](int k, const uint32_t *vals) {
      // lanes S t .. S t + S - 1 of row k: elements S t + N k .. + S - 1
      const int idx = L::S * t + L::NL * k;
      if (idx + L::S <= lim) {
        uint32_t word = 0;
#pragma unroll
        for (int s = 0; s < L::S; ++s) word |= ((vals[s] + base) & L::EMASK) << (E * s);
        out32[idx / L::S] = word;
      } else {
#pragma unroll
        for (int s = 0; s < L::S; ++s)
          if (idx + s < lim) out[idx + s] = (UT)((vals[s] + base) & L::EMASK);
      }
    };
    const bool ok = dispatch_width<E>(w, [&](auto wc) {
      constexpr int W = decltype(wc)::value;
      uint32_t words[W > 0 ? W : 1];
#pragma unroll
      for (int j = 0; j < W; ++j) words[j] = ld_stream_u32(vin + j * 32 + t);
#pragma unroll
      for (int k = 0; k < L::VPL; ++k) {
        uint32_t vals[L::S];
#pragma unroll
        for (int s = 0; s < L::S; ++s) vals[s] = small_value<E, W>(words, s, k);
        emit(k, vals);
      }
    });
    (void)ok;
  }
}

template <int E>
static flsgpu_status decompress_small(const flsgpu_bp_column *bp, const void *bases,
                                      size_t n_values, void *d_out, const flsgpu_decode_opts *o,
                                      flsgpu_stream stream) {
  flsgpu_status s = check_opts(o);
  if (s) return s;
  SmallParams p{};
  p.n_values = n_values;
  p.n_vecs = vecs_of(n_values);
  if (p.n_vecs == 0) return FLSGPU_OK;
  if (!bp->bit_widths || !bp->vector_offsets)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null bit_widths / vector_offsets");
  if (!d_out) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null output");
  if (((uintptr_t)d_out % 4) != 0 || ((uintptr_t)bp->packed_array % 4) != 0)
    return set_error(FLSGPU_ERR_MISALIGNED, "packed words and output must be 4-byte aligned");
  p.packed = reinterpret_cast<const uint32_t *>(bp->packed_array);
  p.bw = bp->bit_widths;
  p.offs = bp->vector_offsets;
  p.bases = bases;
  p.d_status = o ? o->d_status : nullptr;
  p.out = d_out;
  p.n_packed = o ? o->n_packed_values : 0;
  static int bps = 0;
  if (bps == 0) {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_store_small<E>, 256, 0);
    bps = b > 0 ? b : 1;
  }
  const unsigned grid = persistent_blocks(p.n_vecs, 8, bps);
  k_store_small<E><<<grid, 256, 0, (cudaStream_t)stream>>>(p);
  note_launch();
  return check_cuda(cudaGetLastError(), "small-lane decode launch");
}

}  // namespace flsb200

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_decompress_bp_u8(const flsgpu_bp_column *c, uint8_t *o,
                                      const flsgpu_decode_opts *op, flsgpu_stream s) {
  if (!c) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  return decompress_small<8>(c, nullptr, c->n_values, o, op, s);
}
flsgpu_status flsgpu_decompress_bp_u16(const flsgpu_bp_column *c, uint16_t *o,
                                       const flsgpu_decode_opts *op, flsgpu_stream s) {
  if (!c) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  return decompress_small<16>(c, nullptr, c->n_values, o, op, s);
}
flsgpu_status flsgpu_decompress_ffor_u8(const flsgpu_ffor_column *c, uint8_t *o,
                                        const flsgpu_decode_opts *op, flsgpu_stream s) {
  if (!c) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  if (vecs_of(c->n_values) && !c->bases) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null bases");
  return decompress_small<8>(&c->bp, c->bases, c->n_values, o, op, s);
}
flsgpu_status flsgpu_decompress_ffor_u16(const flsgpu_ffor_column *c, uint16_t *o,
                                         const flsgpu_decode_opts *op, flsgpu_stream s) {
  if (!c) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  if (vecs_of(c->n_values) && !c->bases) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null bases");
  return decompress_small<16>(&c->bp, c->bases, c->n_values, o, op, s);
}

}  // extern "C"
