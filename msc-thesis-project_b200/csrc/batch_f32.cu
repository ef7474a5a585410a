// batch_f32.cu -- the batched decode kernels of float columns (see batch.cuh).
#include "batch.cuh"

namespace flsb200 {

flsgpu_status launch_batch_f32(const BatchEntry *table, const size_t *prefix, int n_cols,
                               size_t total_vecs, unsigned long long *counter, cudaStream_t s,
                               int alpx) {
  if (alpx) return BatchLauncher<float, K_ALPX>::launch(table, prefix, n_cols, total_vecs, counter, s);
  return BatchLauncher<float, K_ALP>::launch(table, prefix, n_cols, total_vecs, counter, s);
}

}  // namespace flsb200
