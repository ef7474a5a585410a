// batch_u32.cu -- the batched decode kernels of uint32_t columns (see batch.cuh).
#include "batch.cuh"

namespace flsb200 {

flsgpu_status launch_batch_u32(const BatchEntry *table, const size_t *prefix, int n_cols,
                               size_t total_vecs, unsigned long long *counter, cudaStream_t s,
                               int alpx) {
  (void)alpx;
  return BatchLauncher<uint32_t, K_FFOR>::launch(table, prefix, n_cols, total_vecs, counter, s);
}

}  // namespace flsb200
