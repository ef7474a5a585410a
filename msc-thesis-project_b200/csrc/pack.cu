// pack.cu -- FastLanes bit-packing on the GPU, the encoder side of the
// decode path: FFOR (frame of reference) and BP packing of u16 / u32 / u64
// columns into the reference's interleaved layout (fls::pack,
// src/fls/pack.cpp:29731; fls::ffor, src/fls/ffor.cpp:29861; the base and
// width rule of analyze_ffor, src/alp/encoder.hpp:104-115).
//
// Three launches: k_pack_analyze (per vector: base and bit width), a
// single-block scan of the vectors' packed sizes, and k_pack_write.  One warp
// per vector; every thread owns 32 values of the vector and writes the
// 32 * w bits they occupy in their lane's bit stream:
//   u32: thread t = lane t, values k = 0..31 (element t + 32k), stream words
//        0..w-1 of lane t (32-bit words at packed[j*32 + t]);
//   u64: thread t = half t/16 of lane t%16, values 32h..32h+31 (element
//        l + 16k); the half's 32w bits are exactly the 32-bit words
//        h*w .. h*w+w-1 of the lane's stream (the low / high halves of the
//        64-bit words at packed[j*16 + l]);
//   u16: thread t = lanes 2t and 2t+1, 16 values each (element lane + 64j);
//        16-bit stream words 0..w-1 of each lane at packed[j*64 + lane];
//   u8:  thread t = lanes 4t .. 4t+3, 8 values each (element lane + 128j);
//        8-bit stream words 0..w-1 of each lane at packed[j*128 + lane].
// A value occupies bits [k*w, (k+1)*w) of its lane's stream, least
// significant bit first, so the words decode with flsgpu_decompress_*.
#include "common.cuh"

namespace flsb200 {

// Value k (0..31) owned by thread t of a vector.
template <typename U> __device__ __forceinline__ size_t owned_index(int t, int k) {
  if constexpr (sizeof(U) == 4) {
    return (size_t)t + 32u * k;
  } else if constexpr (sizeof(U) == 8) {
    return (size_t)(t & 15) + 16u * (32u * (t >> 4) + k);
  } else if constexpr (sizeof(U) == 2) {
    return (size_t)(2 * t + (k >> 4)) + 64u * (k & 15);
  } else {
    return (size_t)(4 * t + (k >> 3)) + 128u * (k & 7);
  }
}

__device__ __forceinline__ uint64_t shfl_xor_u64(uint64_t v, int m) {
  const uint32_t lo = __shfl_xor_sync(0xffffffffu, (uint32_t)v, m);
  const uint32_t hi = __shfl_xor_sync(0xffffffffu, (uint32_t)(v >> 32), m);
  return ((uint64_t)hi << 32) | lo;
}

// Per vector: base (mode 0 unsigned minimum, 1 signed minimum, 2 zero) and
// width = bits of (max - base) in the type's unsigned arithmetic.
template <typename U>
__global__ void __launch_bounds__(256) k_pack_analyze(const U *__restrict__ vals, size_t n_vecs,
                                                      int mode, uint8_t *bw, U *bases) {
  constexpr int BITS = (int)sizeof(U) * 8;
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const U *vec = vals + v * VEC;
    // keys: the values mapped so that unsigned order of the key is the
    // order the mode asks for (signed: flip the sign bit)
    const uint64_t flip = mode == 1 ? (1ull << (BITS - 1)) : 0ull;
    uint64_t kmin = ~0ull, kmax = 0;
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      const uint64_t key = (uint64_t)vec[owned_index<U>(t, k)] ^ flip;
      kmin = key < kmin ? key : kmin;
      kmax = key > kmax ? key : kmax;
    }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
      const uint64_t a = shfl_xor_u64(kmin, m), b = shfl_xor_u64(kmax, m);
      kmin = a < kmin ? a : kmin;
      kmax = b > kmax ? b : kmax;
    }
    const U vmin = (U)(kmin ^ flip), vmax = (U)(kmax ^ flip);
    const U base = mode == 2 ? (U)0 : vmin;
    const U range = (U)(vmax - base);
    const int w = range == 0 ? 0 : BITS - (sizeof(U) == 8 ? __clzll((long long)range)
                                                          : __clz((int)(uint32_t)range) - (32 - BITS));
    if (t == 0) {
      bw[v] = (uint8_t)w;
      if (bases) bases[v] = base;
    }
  }
}

// Exclusive scan of packed sizes (bw * lanes words) in one block.
__global__ void __launch_bounds__(1024) k_pack_scan(const uint8_t *bw, size_t n, int lanes,
                                                    uint64_t *offs, uint64_t *total) {
  __shared__ uint64_t s[1024];
  const int tid = threadIdx.x;
  const size_t per = (n + 1023) / 1024;
  const size_t lo = tid * per, hi = lo + per < n ? lo + per : n;
  uint64_t sum = 0;
  for (size_t i = lo; i < hi; ++i) sum += (uint64_t)bw[i] * lanes;
  s[tid] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const uint64_t a = tid >= o ? s[tid - o] : 0;
    __syncthreads();
    s[tid] += a;
    __syncthreads();
  }
  uint64_t r = s[tid] - sum;
  for (size_t i = lo; i < hi; ++i) {
    offs[i] = r;
    r += (uint64_t)bw[i] * lanes;
  }
  if (tid == 1023 && total) *total = s[1023];
}

// LSB-first bit stream of E-bit words (E = 32 or 16).
template <int E> struct BitWriter {
  uint64_t acc = 0;
  int fill = 0;
  int word = 0;
  // n <= 32 bits of v (v < 2^n)
  template <typename Emit> __device__ __forceinline__ void put(uint64_t v, int n, Emit &&emit) {
    acc |= v << fill;
    fill += n;
    while (fill >= E) {
      emit(word++, (uint32_t)(acc & ((1ull << E) - 1)));
      acc >>= E;
      fill -= E;
    }
  }
};

template <typename U>
__global__ void __launch_bounds__(256) k_pack_write(const U *__restrict__ vals, size_t n_vecs,
                                                    const uint8_t *__restrict__ bw,
                                                    const U *__restrict__ bases,
                                                    const uint64_t *__restrict__ offs, U *packed) {
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const U *vec = vals + v * VEC;
    const int w = bw[v];
    if (w == 0) continue;
    const U base = bases ? bases[v] : (U)0;
    U *out = packed + offs[v];
    if constexpr (sizeof(U) == 4) {
      BitWriter<32> bwr;
      auto emit = [&](int i, uint32_t x) { out[(size_t)i * 32 + t] = x; };
      for (int k = 0; k < 32; ++k) bwr.put((uint32_t)(vec[owned_index<U>(t, k)] - base), w, emit);
    } else if constexpr (sizeof(U) == 8) {
      const int l = t & 15, h = t >> 4;
      uint32_t *o32 = reinterpret_cast<uint32_t *>(out);
      BitWriter<32> bwr;
      auto emit = [&](int i, uint32_t x) {
        const int j = h * w + i;  // 32-bit word of the lane's stream
        o32[2 * ((size_t)(j >> 1) * 16 + l) + (j & 1)] = x;
      };
      for (int k = 0; k < 32; ++k) {
        const uint64_t d = (uint64_t)(vec[owned_index<U>(t, k)] - base);
        if (w <= 32) {
          bwr.put(d, w, emit);
        } else {
          bwr.put(d & 0xFFFFFFFFull, 32, emit);
          bwr.put(d >> 32, w - 32, emit);
        }
      }
    } else if constexpr (sizeof(U) == 2) {
      for (int half = 0; half < 2; ++half) {
        const int lane = 2 * t + half;
        BitWriter<16> bwr;
        auto emit = [&](int i, uint32_t x) { out[(size_t)i * 64 + lane] = (U)x; };
        for (int j = 0; j < 16; ++j) bwr.put((uint16_t)(vec[(size_t)lane + 64u * j] - base), w, emit);
      }
    } else {
      // u8: thread t = lanes 4t .. 4t + 3, 8 values each (element lane + 128 j)
      for (int q = 0; q < 4; ++q) {
        const int lane = 4 * t + q;
        BitWriter<8> bwr;
        auto emit = [&](int i, uint32_t x) { out[(size_t)i * 128 + lane] = (U)x; };
        for (int j = 0; j < 8; ++j) bwr.put((uint8_t)(vec[(size_t)lane + 128u * j] - base), w, emit);
      }
    }
  }
}

template <typename U>
static flsgpu_status pack_column(const U *vals, size_t n_values, uint32_t mode, U *packed,
                                 uint8_t *bw, uint64_t *offs, U *bases, uint64_t *n_packed,
                                 flsgpu_stream stream) {
  if (!vals || !packed || !bw || !offs || (n_values % VEC) || mode > 2 ||
      (mode != 2 && !bases))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT,
                     "pack: null array, n_values not a multiple of 1024, or bad base mode");
  const size_t n_vecs = n_values / VEC;
  if (!n_vecs) return FLSGPU_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned grid = persistent_blocks(n_vecs, 8, 4);
  k_pack_analyze<U><<<grid, 256, 0, s>>>(vals, n_vecs, (int)mode, bw, mode == 2 ? nullptr : bases);
  k_pack_scan<<<1, 1024, 0, s>>>(bw, n_vecs, VEC / (int)(sizeof(U) * 8), offs, n_packed);
  k_pack_write<U><<<grid, 256, 0, s>>>(vals, n_vecs, bw, mode == 2 ? nullptr : bases, offs, packed);
  note_launch(3);
  return check_cuda(cudaGetLastError(), "pack");
}

}  // namespace flsb200

using namespace flsb200;

extern "C" {
flsgpu_status flsgpu_ffor_encode_u8(const uint8_t *d_values, size_t n_values, uint32_t base_mode,
                                    uint8_t *d_packed, uint8_t *d_bit_widths,
                                    uint64_t *d_vector_offsets, uint8_t *d_bases,
                                    uint64_t *d_n_packed, flsgpu_stream stream) {
  return pack_column<uint8_t>(d_values, n_values, base_mode, d_packed, d_bit_widths,
                              d_vector_offsets, d_bases, d_n_packed, stream);
}
flsgpu_status flsgpu_ffor_encode_u16(const uint16_t *d_values, size_t n_values, uint32_t base_mode,
                                     uint16_t *d_packed, uint8_t *d_bit_widths,
                                     uint64_t *d_vector_offsets, uint16_t *d_bases,
                                     uint64_t *d_n_packed, flsgpu_stream stream) {
  return pack_column<uint16_t>(d_values, n_values, base_mode, d_packed, d_bit_widths,
                               d_vector_offsets, d_bases, d_n_packed, stream);
}
flsgpu_status flsgpu_ffor_encode_u32(const uint32_t *d_values, size_t n_values, uint32_t base_mode,
                                     uint32_t *d_packed, uint8_t *d_bit_widths,
                                     uint64_t *d_vector_offsets, uint32_t *d_bases,
                                     uint64_t *d_n_packed, flsgpu_stream stream) {
  return pack_column<uint32_t>(d_values, n_values, base_mode, d_packed, d_bit_widths,
                               d_vector_offsets, d_bases, d_n_packed, stream);
}
flsgpu_status flsgpu_ffor_encode_u64(const uint64_t *d_values, size_t n_values, uint32_t base_mode,
                                     uint64_t *d_packed, uint8_t *d_bit_widths,
                                     uint64_t *d_vector_offsets, uint64_t *d_bases,
                                     uint64_t *d_n_packed, flsgpu_stream stream) {
  return pack_column<uint64_t>(d_values, n_values, base_mode, d_packed, d_bit_widths,
                               d_vector_offsets, d_bases, d_n_packed, stream);
}
}
