// capi.cu -- library-wide state: error strings, constants, device info.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "common.cuh"
#include "autotune_table.h"

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

// ---- decode tuning ------------------------------------------------------
// Variant per (value type, kind); prefetch masks per lane width.  Defaults:
// the compiled table (autotune_table.h).
static std::atomic<uint8_t> g_variant[4][4] = {};
static std::atomic<uint64_t> g_prefetch[2][2];
static std::once_flag g_tuning_once;

static void tuning_defaults() {
  for (int t = 0; t < 4; ++t)
    for (int k = 0; k < 4; ++k) g_variant[t][k].store(tuned::kVariant[t][k]);
  uint64_t m32[2] = {0, 0}, m64[2] = {0, 0};
  for (int w = 0; w <= 32; ++w)
    if (tuned::kPrefetch32[w]) m32[w >> 6] |= 1ull << (w & 63);
  for (int w = 0; w <= 64; ++w)
    if (tuned::kPrefetch64[w]) m64[w >> 6] |= 1ull << (w & 63);
  g_prefetch[0][0].store(m32[0]);
  g_prefetch[0][1].store(m32[1]);
  g_prefetch[1][0].store(m64[0]);
  g_prefetch[1][1].store(m64[1]);
}

int tuned_variant(int type, int kind) {
  std::call_once(g_tuning_once, tuning_defaults);
  return g_variant[type & 3][kind & 3].load(std::memory_order_relaxed);
}

void tuned_prefetch(int lane_bits, uint64_t out[2]) {
  std::call_once(g_tuning_once, tuning_defaults);
  const int i = lane_bits == 64 ? 1 : 0;
  out[0] = g_prefetch[i][0].load(std::memory_order_relaxed);
  out[1] = g_prefetch[i][1].load(std::memory_order_relaxed);
}

}  // namespace flsb200

extern "C" {
uint32_t flsgpu_abi_version(void) { return FLSGPU_B200_ABI_VERSION; }
const char *flsgpu_last_error(void) { return flsb200::g_err; }
uint64_t flsgpu_launch_count(void) { return flsb200::g_launches.load(); }
}

extern "C" {
flsgpu_status flsgpu_tuning_set_variant(uint32_t type, uint32_t kind, uint32_t variant) {
  using namespace flsb200;
  if (type > 3 || kind > 3 || variant == FLSGPU_VARIANT_AUTO || variant >= FLSGPU_VARIANT_COUNT)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "tuning: type %u kind %u variant %u", type,
                     kind, variant);
  std::call_once(g_tuning_once, tuning_defaults);
  g_variant[type][kind].store((uint8_t)variant);
  return FLSGPU_OK;
}
flsgpu_status flsgpu_tuning_get_variant(uint32_t type, uint32_t kind, uint32_t *variant) {
  using namespace flsb200;
  if (type > 3 || kind > 3 || !variant)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "tuning: type %u kind %u", type, kind);
  *variant = (uint32_t)tuned_variant((int)type, (int)kind);
  return FLSGPU_OK;
}
flsgpu_status flsgpu_tuning_set_prefetch(uint32_t lane_bits, const uint64_t mask[2]) {
  using namespace flsb200;
  if ((lane_bits != 32 && lane_bits != 64) || !mask)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "tuning: lane width %u", lane_bits);
  std::call_once(g_tuning_once, tuning_defaults);
  const int i = lane_bits == 64 ? 1 : 0;
  g_prefetch[i][0].store(mask[0]);
  g_prefetch[i][1].store(mask[1]);
  return FLSGPU_OK;
}
flsgpu_status flsgpu_tuning_get_prefetch(uint32_t lane_bits, uint64_t mask[2]) {
  using namespace flsb200;
  if ((lane_bits != 32 && lane_bits != 64) || !mask)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "tuning: lane width %u", lane_bits);
  tuned_prefetch((int)lane_bits, mask);
  return FLSGPU_OK;
}
}
