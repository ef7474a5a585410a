// device_api_kernels.cu -- test program for the device-side decoders
// (include/flsgpu_b200_device.cuh): user kernels written the way the
// reference's kernels::device::decompress_column is (src/engine/kernels.cuh:
// 13-32: one thread per FastLanes lane, N_LANES threads per vector, a
// Decompressor per thread and unpack_next_into into registers, written to
// global memory at lane + (i + j) * N_LANES), exported as C launchers for the
// parity tests.  Each launcher returns the CUDA error code (0 = success).
#include "flsgpu_b200_device.cuh"

using namespace flsgpu_b200::device;

template <typename T, unsigned NV, typename Dec, typename Col>
__global__ void k_user_decode(const Col col, size_t n_vecs, T *out) {
  constexpr unsigned N = lane_traits<T>::N_LANES;
  const unsigned lane = threadIdx.x % N;
  const size_t v = (size_t)blockIdx.x * (blockDim.x / N) + threadIdx.x / N;
  if (v >= n_vecs) return;
  Dec d(col, v, lane);
  T regs[NV];
  T *o = out + v * 1024;
  for (unsigned i = 0; i < values_per_lane<T>(); i += NV) {
    d.unpack_next_into(regs);
#pragma unroll
    for (unsigned j = 0; j < NV; ++j) o[lane + (i + j) * N] = regs[j];
  }
}

template <typename T, template <typename, unsigned> class Dec, typename Col>
static int launch(const Col *c, T *out, unsigned nv) {
  const size_t n_vecs = (c->n_values + 1023) / 1024;
  const unsigned threads = 128, per_block = threads / lane_traits<T>::N_LANES;
  const unsigned blocks = (unsigned)((n_vecs + per_block - 1) / per_block);
  if (nv == 4)
    k_user_decode<T, 4, Dec<T, 4>, Col><<<blocks, threads>>>(*c, n_vecs, out);
  else
    k_user_decode<T, 1, Dec<T, 1>, Col><<<blocks, threads>>>(*c, n_vecs, out);
  return (int)cudaDeviceSynchronize();
}

extern "C" {
int user_decode_bp_u32(const flsgpu_bp_column *c, uint32_t *o, unsigned nv) { return launch<uint32_t, BPDecompressor>(c, o, nv); }
int user_decode_bp_u64(const flsgpu_bp_column *c, uint64_t *o, unsigned nv) { return launch<uint64_t, BPDecompressor>(c, o, nv); }
int user_decode_ffor_u32(const flsgpu_ffor_column *c, uint32_t *o, unsigned nv) { return launch<uint32_t, FFORDecompressor>(c, o, nv); }
int user_decode_ffor_u64(const flsgpu_ffor_column *c, uint64_t *o, unsigned nv) { return launch<uint64_t, FFORDecompressor>(c, o, nv); }
int user_decode_alp_f32(const flsgpu_alp_column *c, float *o, unsigned nv) { return launch<float, ALPDecompressor>(c, o, nv); }
int user_decode_alp_f64(const flsgpu_alp_column *c, double *o, unsigned nv) { return launch<double, ALPDecompressor>(c, o, nv); }
int user_decode_alpx_f32(const flsgpu_alpx_column *c, float *o, unsigned nv) { return launch<float, ALPExtendedDecompressor>(c, o, nv); }
int user_decode_alpx_f64(const flsgpu_alpx_column *c, double *o, unsigned nv) { return launch<double, ALPExtendedDecompressor>(c, o, nv); }
}
