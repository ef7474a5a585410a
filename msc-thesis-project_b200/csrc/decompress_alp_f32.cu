// decompress_alp_f32.cu -- C ABI: full decompression of one column type
// (kernels::device::decompress_column with ALPDecompressor, src/flsgpu/alp.cuh:463-485).  One translation unit per
// entry point, so that the per-width decode kernels of the library build in
// parallel.
#include "kernels.cuh"

using namespace flsb200;

extern "C" flsgpu_status flsgpu_decompress_alp_f32(const flsgpu_alp_column *c, float *o,
                                                 const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<float, K_ALP>(c, o, op, s);
}
