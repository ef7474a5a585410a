// batch_f64.cu -- k_batch<double> (see batch.cuh).
#include "batch.cuh"

namespace flsb200 {

flsgpu_status launch_batch_f64(const BatchEntry *table, const size_t *prefix, int n_cols,
                               size_t total_vecs, unsigned long long *counter, cudaStream_t s) {
  flsgpu_status st = check_cuda(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s), "memset");
  if (st) return st;
  const unsigned grid = persistent_blocks(total_vecs ? total_vecs : 1, 8,
                                          BatchLauncher<double>::blocks_per_sm());
  k_batch<double><<<grid, 256, 0, s>>>(table, prefix, n_cols, counter);
  note_launch();
  return check_cuda(cudaGetLastError(), "k_batch launch");
}

}  // namespace flsb200
