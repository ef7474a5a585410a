// capi.cu -- library-wide state: error strings, constants, device info.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "common.cuh"

namespace flsb200 {

static thread_local char g_err[512] = "";
static std::atomic<uint64_t> g_launches{0};

flsgpu_status set_error(flsgpu_status s, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return s;
}

flsgpu_status check_cuda(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return FLSGPU_OK;
  if (e == cudaErrorMemoryAllocation)
    return set_error(FLSGPU_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
  return set_error(FLSGPU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int sm_count() {
  int dev = 0;
  cudaGetDevice(&dev);
  static int cached[64] = {0};
  if (dev < 0 || dev >= 64) dev = 0;
  if (cached[dev] == 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = n > 0 ? n : 1;
  }
  return cached[dev];
}

void note_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

}  // namespace flsb200

extern "C" {
uint32_t flsgpu_abi_version(void) { return FLSGPU_B200_ABI_VERSION; }
const char *flsgpu_last_error(void) { return flsb200::g_err; }
uint64_t flsgpu_launch_count(void) { return flsb200::g_launches.load(); }
}
