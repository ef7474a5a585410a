// decompress_bp_u32.cu -- C ABI: full decompression of one column type
// (kernels::device::decompress_column, src/engine/kernels.cuh:13-32).  One translation unit per
// entry point, so that the per-width decode kernels of the library build in
// parallel.
#include "kernels.cuh"

using namespace flsb200;

extern "C" flsgpu_status flsgpu_decompress_bp_u32(const flsgpu_bp_column *c, uint32_t *o,
                                                 const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<uint32_t, K_BP>(c, o, op, s);
}
