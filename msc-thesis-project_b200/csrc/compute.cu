// compute.cu -- C ABI: synthetic ALU load after decoding (kernels::device::compute_column,
// src/engine/kernels.cuh:56-89).
#include <cstring>

#include "kernels.cuh"

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_compute_ffor_u32(const flsgpu_ffor_column *c, uint32_t n, uint8_t *o,
                                      const flsgpu_decode_opts *op, flsgpu_stream s) {
  return compute<uint32_t>(c, n, o, op, s);
}

flsgpu_status flsgpu_compute_ffor_u64(const flsgpu_ffor_column *c, uint32_t n, uint8_t *o,
                                      const flsgpu_decode_opts *op, flsgpu_stream s) {
  return compute<uint64_t>(c, n, o, op, s);
}

}  // extern "C"
