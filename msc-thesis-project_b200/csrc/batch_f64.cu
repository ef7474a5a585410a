// batch_f64.cu -- the batched decode kernels of double columns (see batch.cuh).
#include "batch.cuh"

namespace flsb200 {

flsgpu_status launch_batch_f64(const BatchEntry *table, const size_t *prefix, int n_cols,
                               size_t total_vecs, unsigned long long *counter, cudaStream_t s,
                               int alpx) {
  if (alpx) return BatchLauncher<double, K_ALPX>::launch(table, prefix, n_cols, total_vecs, counter, s);
  return BatchLauncher<double, K_ALP>::launch(table, prefix, n_cols, total_vecs, counter, s);
}

}  // namespace flsb200
