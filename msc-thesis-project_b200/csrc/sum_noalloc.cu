// sum_noalloc.cu -- the f64 ALP decode-and-sum without any allocation.
//
// flsgpu_sum_alp_f64 needs scratch for the per-vector partial sums of its
// fixed reduction tree and takes it from the caller (d_partials).  Some
// callers cannot hand out device memory at all: a query engine that runs
// operators inside a fixed memory budget it manages itself, a host thread
// that is capturing a CUDA graph (cudaMalloc is not allowed while a stream
// is being captured in the global or thread-local mode), or a plug-in
// loaded into a process whose allocator it must not touch.  For them this
// entry point keeps the scratch in a statically sized array in device
// memory, reserved when the library is loaded on a GPU and held until the
// process exits, so a call needs no cudaMalloc, cudaFree or library
// allocation.
//
// Limits and sharing: the array holds the partials of at most
// FLSGPU_NOALLOC_MAX_VECTORS vectors (2^18 vectors, 2^28 values, 2 MiB);
// larger columns are rejected.  Every call on a device uses the same array,
// so calls whose kernels overlap on the GPU (different streams, or several
// host threads) race on it; serialise them.  Each call overwrites every
// partial it reads (a vector rejected by the metadata checks writes +0.0),
// so stale contents from an earlier call never leak into a result and
// nothing has to be cleared.
//
// The device address is cached per device index for the life of the
// process.  cudaDeviceReset (or anything else that destroys the primary
// context) reloads the module and invalidates it, so the cache is keyed by
// the context as well: a call made in a different context than the one
// the address was taken in looks it up again.
#include <cuda.h>

#include <mutex>

#include "kernels.cuh"

namespace flsb200 {

constexpr size_t kNoAllocMaxVectors = FLSGPU_NOALLOC_MAX_VECTORS;
// partials of every vector, then the chunk results of the pairwise tree
constexpr size_t kNoAllocScratch = kNoAllocMaxVectors + (kNoAllocMaxVectors + 2047) / 2048 + 1;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocScratch];

// the decode-and-sum itself (sum.cu)
flsgpu_status sum_alp_f64_impl(const flsgpu_alp_column *c, double *d_sum, double *d_partials,
                               const flsgpu_decode_opts *op, flsgpu_stream s);

// In host code g_noalloc_partials names a host-side stand-in, not device
// memory: its device address is looked up with the device current, and
// cached per device together with the id of the context it was taken in.
static std::mutex g_noalloc_mu;
static double *g_noalloc_addr[64] = {nullptr};
static unsigned long long g_noalloc_ctx[64] = {0};

// Process-unique id of the context current on the calling thread, 0 when
// there is none.  The two driver entry points are looked up through the
// runtime, so the library does not link against the driver library itself
// (it still loads where no GPU driver is installed).
static unsigned long long current_context_id() {
  using get_current_t = CUresult (*)(CUcontext *);
  using get_id_t = CUresult (*)(CUcontext, unsigned long long *);
  static get_current_t get_current = nullptr;
  static get_id_t get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<get_current_t>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<get_id_t>(f);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx ||
      get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

static flsgpu_status noalloc_scratch(double **out) {
  int dev = 0;
  flsgpu_status s = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (s) return s;
  if (dev < 0 || dev >= 64) return set_error(FLSGPU_ERR_UNSUPPORTED, "device index %d", dev);
  // the id of the context current on this thread (0 when the CUDA runtime
  // has not been used on it yet: then the lookup below binds the device's
  // primary context and the id is read afterwards)
  unsigned long long ctx_id = current_context_id();
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev] || ctx_id == 0 || g_noalloc_ctx[dev] != ctx_id) {
    void *p = nullptr;
    s = check_cuda(cudaGetSymbolAddress(&p, g_noalloc_partials), "cudaGetSymbolAddress");
    if (s) return s;
    if ((ctx_id = current_context_id()) == 0)
      return set_error(FLSGPU_ERR_CUDA, "flsgpu_sum_alp_f64_noalloc: no current CUDA context");
    g_noalloc_addr[dev] = static_cast<double *>(p);
    g_noalloc_ctx[dev] = ctx_id;
  }
  *out = g_noalloc_addr[dev];
  return FLSGPU_OK;
}

}  // namespace flsb200

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_sum_alp_f64_noalloc(const flsgpu_alp_column *c, double *d_sum,
                                         const flsgpu_decode_opts *op, flsgpu_stream s) {
  if (!c) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  const size_t n_vecs = vecs_of(c->n_values);
  if (n_vecs > kNoAllocMaxVectors)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT,
                     "flsgpu_sum_alp_f64_noalloc: %zu vectors exceed the static scratch limit of "
                     "%zu vectors (%zu values); use flsgpu_sum_alp_f64 with caller workspace",
                     n_vecs, kNoAllocMaxVectors, kNoAllocMaxVectors * VEC);
  double *scratch = nullptr;
  flsgpu_status st = noalloc_scratch(&scratch);
  if (st) return st;
  return sum_alp_f64_impl(c, d_sum, scratch, op, s);
}

}  // extern "C"
