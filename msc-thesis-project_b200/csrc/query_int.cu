// query_int.cu -- C ABI: magic-value scan of BP / FFOR columns (kernels::device::query_column,
// src/engine/kernels.cuh:34-54).
#include <cstring>

#include "kernels.cuh"

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_query_bp_u32(const flsgpu_bp_column *c, uint32_t m, uint8_t *f,
                                  const flsgpu_decode_opts *op, flsgpu_stream s) {
  return query<uint32_t, K_BP>(c, m, f, op, s);
}

flsgpu_status flsgpu_query_bp_u64(const flsgpu_bp_column *c, uint64_t m, uint8_t *f,
                                  const flsgpu_decode_opts *op, flsgpu_stream s) {
  return query<uint64_t, K_BP>(c, m, f, op, s);
}

flsgpu_status flsgpu_query_ffor_u32(const flsgpu_ffor_column *c, uint32_t m, uint8_t *f,
                                    const flsgpu_decode_opts *op, flsgpu_stream s) {
  return query<uint32_t, K_FFOR>(c, m, f, op, s);
}

flsgpu_status flsgpu_query_ffor_u64(const flsgpu_ffor_column *c, uint64_t m, uint8_t *f,
                                    const flsgpu_decode_opts *op, flsgpu_stream s) {
  return query<uint64_t, K_FFOR>(c, m, f, op, s);
}

}  // extern "C"
