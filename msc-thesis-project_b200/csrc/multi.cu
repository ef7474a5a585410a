// multi.cu -- C ABI: multi-column conjunctive scan (multi_column::query_multi_column,
// src/generated-bindings/multi-column-device-kernels.cuh:11-439).
#include <cstring>

#include "kernels.cuh"

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_query_multi_column_ffor_u32(const flsgpu_ffor_column *c, uint32_t n,
                                                 uint32_t v, uint8_t *o,
                                                 const flsgpu_decode_opts *op, flsgpu_stream s) {
  return multi<uint32_t, K_FFOR>(c, n, v, o, op, s);
}

flsgpu_status flsgpu_query_multi_column_ffor_u64(const flsgpu_ffor_column *c, uint32_t n,
                                                 uint64_t v, uint8_t *o,
                                                 const flsgpu_decode_opts *op, flsgpu_stream s) {
  return multi<uint64_t, K_FFOR>(c, n, v, o, op, s);
}

flsgpu_status flsgpu_query_multi_column_alp_f32(const flsgpu_alp_column *c, uint32_t n, float v,
                                                uint8_t *o, const flsgpu_decode_opts *op,
                                                flsgpu_stream s) {
  return multi<float, K_ALP>(c, n, v, o, op, s);
}

flsgpu_status flsgpu_query_multi_column_alp_f64(const flsgpu_alp_column *c, uint32_t n, double v,
                                                uint8_t *o, const flsgpu_decode_opts *op,
                                                flsgpu_stream s) {
  return multi<double, K_ALP>(c, n, v, o, op, s);
}

}  // extern "C"
