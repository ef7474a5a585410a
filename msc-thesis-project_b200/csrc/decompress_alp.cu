// decompress_alp.cu -- C ABI: full decompression of ALP / ALP-extended columns (kernels::device::
// decompress_column with ALPDecompressor, src/flsgpu/alp.cuh:463-485).
#include <cstring>

#include "kernels.cuh"

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_decompress_alp_f32(const flsgpu_alp_column *c, float *o,
                                        const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<float, K_ALP>(c, o, op, s);
}

flsgpu_status flsgpu_decompress_alp_f64(const flsgpu_alp_column *c, double *o,
                                        const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<double, K_ALP>(c, o, op, s);
}

flsgpu_status flsgpu_decompress_alpx_f32(const flsgpu_alpx_column *c, float *o,
                                         const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<float, K_ALPX>(c, o, op, s);
}

flsgpu_status flsgpu_decompress_alpx_f64(const flsgpu_alpx_column *c, double *o,
                                         const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<double, K_ALPX>(c, o, op, s);
}

}  // extern "C"
