// query_alp.cu -- C ABI: magic-value scan of ALP / ALP-extended columns (kernels::device::
// query_column with ALPDecompressor, src/engine/kernels.cuh:34-54).
#include <cstring>

#include "kernels.cuh"

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_query_alp_f32(const flsgpu_alp_column *c, float m, uint8_t *f,
                                   const flsgpu_decode_opts *op, flsgpu_stream s) {
  return query<float, K_ALP>(c, m, f, op, s);
}

flsgpu_status flsgpu_query_alp_f64(const flsgpu_alp_column *c, double m, uint8_t *f,
                                   const flsgpu_decode_opts *op, flsgpu_stream s) {
  return query<double, K_ALP>(c, m, f, op, s);
}

flsgpu_status flsgpu_query_alpx_f32(const flsgpu_alpx_column *c, float m, uint8_t *f,
                                    const flsgpu_decode_opts *op, flsgpu_stream s) {
  return query<float, K_ALPX>(c, m, f, op, s);
}

flsgpu_status flsgpu_query_alpx_f64(const flsgpu_alpx_column *c, double m, uint8_t *f,
                                    const flsgpu_decode_opts *op, flsgpu_stream s) {
  return query<double, K_ALPX>(c, m, f, op, s);
}

}  // extern "C"
