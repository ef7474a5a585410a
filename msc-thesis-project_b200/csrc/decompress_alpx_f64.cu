// decompress_alpx_f64.cu -- C ABI: full decompression of one column type
// (kernels::device::decompress_column with ALPDecompressor, src/flsgpu/alp.cuh:463-485).  One translation unit per
// entry point, so that the per-width decode kernels of the library build in
// parallel.
#include "kernels.cuh"

using namespace flsb200;

extern "C" flsgpu_status flsgpu_decompress_alpx_f64(const flsgpu_alpx_column *c, double *o,
                                                 const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<double, K_ALPX>(c, o, op, s);
}
