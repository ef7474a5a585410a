// sum.cu -- C ABI: decode fused with a sum reduction.
#include <cstring>

#include "kernels.cuh"

namespace flsb200 {
// The f64 ALP decode-and-sum, shared with the allocation-free entry point
// (sum_noalloc.cu), which passes its static scratch as the partials.
flsgpu_status sum_alp_f64_impl(const flsgpu_alp_column *c, double *d_sum, double *d_partials,
                               const flsgpu_decode_opts *op, flsgpu_stream s) {
  return sum_f64<K_ALP>(c, d_sum, d_partials, op, s);
}
}  // namespace flsb200

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_sum_ffor_u32(const flsgpu_ffor_column *c, uint64_t *d_sum,
                                  const flsgpu_decode_opts *op, flsgpu_stream s) {
  return sum_int<uint32_t>(c, d_sum, op, s);
}

flsgpu_status flsgpu_sum_ffor_u64(const flsgpu_ffor_column *c, uint64_t *d_sum,
                                  const flsgpu_decode_opts *op, flsgpu_stream s) {
  return sum_int<uint64_t>(c, d_sum, op, s);
}

flsgpu_status flsgpu_sum_alp_f64(const flsgpu_alp_column *c, double *d_sum, double *d_partials,
                                 const flsgpu_decode_opts *op, flsgpu_stream s) {
  return sum_alp_f64_impl(c, d_sum, d_partials, op, s);
}

flsgpu_status flsgpu_sum_alpx_f64(const flsgpu_alpx_column *c, double *d_sum, double *d_partials,
                                  const flsgpu_decode_opts *op, flsgpu_stream s) {
  return sum_f64<K_ALPX>(c, d_sum, d_partials, op, s);
}

size_t flsgpu_sum_workspace_f64(size_t n_values) {
  const size_t n_vecs = (n_values + 1023) / 1024;
  return n_vecs + (n_vecs + 2047) / 2048 + 1;
}

}  // extern "C"
