// decompress_int.cu -- C ABI: full decompression of BP / FFOR columns (kernels::device::decompress_column,
// src/engine/kernels.cuh:13-32).
#include <cstring>

#include "kernels.cuh"

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_decompress_bp_u32(const flsgpu_bp_column *c, uint32_t *o,
                                       const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<uint32_t, K_BP>(c, o, op, s);
}

flsgpu_status flsgpu_decompress_bp_u64(const flsgpu_bp_column *c, uint64_t *o,
                                       const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<uint64_t, K_BP>(c, o, op, s);
}

flsgpu_status flsgpu_decompress_ffor_u32(const flsgpu_ffor_column *c, uint32_t *o,
                                         const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<uint32_t, K_FFOR>(c, o, op, s);
}

flsgpu_status flsgpu_decompress_ffor_u64(const flsgpu_ffor_column *c, uint64_t *o,
                                         const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<uint64_t, K_FFOR>(c, o, op, s);
}

}  // extern "C"
