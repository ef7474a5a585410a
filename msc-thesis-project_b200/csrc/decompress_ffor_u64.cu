// decompress_ffor_u64.cu -- C ABI: full decompression of one column type
// (kernels::device::decompress_column, src/engine/kernels.cuh:13-32).  One translation unit per
// entry point, so that the per-width decode kernels of the library build in
// parallel.
#include "kernels.cuh"

using namespace flsb200;

extern "C" flsgpu_status flsgpu_decompress_ffor_u64(const flsgpu_ffor_column *c, uint64_t *o,
                                                 const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress<uint64_t, K_FFOR>(c, o, op, s);
}
