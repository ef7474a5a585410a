// common.cuh -- shared definitions of the B200 FastLanes/ALP kernels.
//
// Geometry (reference src/flsgpu/utils.cuh:75-86): a vector is 1024 values;
// a T-bit type has N_LANES = 1024/bits(T) lanes of bits(T) values; value k
// of lane l is element l + k*N_LANES; packed word j of lane l sits at
// packed[j*N_LANES + l]; a vector packed at width w occupies w*N_LANES words.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/flsgpu_b200.h"

namespace flsb200 {

constexpr int VEC = 1024;
constexpr int WARP = 32;

template <typename U> struct Lanes {
  static constexpr int BITS = sizeof(U) * 8;
  static constexpr int N = VEC / BITS;  // lanes per vector
};

// ALP tables, one copy per translation unit (reference src/alp/constants.hpp:49-55 float, :76-144 double).
static __constant__ float c_f32_frac[11] = {1.0f,  0.1f,  0.01f, 0.001f, 0.0001f, 1e-5f,
                                     1e-6f, 1e-7f, 1e-8f, 1e-9f,  1e-10f};
static __constant__ int32_t c_f32_fact[10] = {1,      10,      100,      1000,      10000,
                                       100000, 1000000, 10000000, 100000000, 1000000000};
static __constant__ double c_f64_frac[21] = {1.0,   0.1,   0.01,  0.001, 0.0001, 1e-5,  1e-6,
                                      1e-7,  1e-8,  1e-9,  1e-10, 1e-11,  1e-12, 1e-13,
                                      1e-14, 1e-15, 1e-16, 1e-17, 1e-18,  1e-19, 1e-20};
static __constant__ int64_t c_f64_fact[19] = {1LL,
                                       10LL,
                                       100LL,
                                       1000LL,
                                       10000LL,
                                       100000LL,
                                       1000000LL,
                                       10000000LL,
                                       100000000LL,
                                       1000000000LL,
                                       10000000000LL,
                                       100000000000LL,
                                       1000000000000LL,
                                       10000000000000LL,
                                       100000000000000LL,
                                       1000000000000000LL,
                                       10000000000000000LL,
                                       100000000000000000LL,
                                       1000000000000000000LL};

// ---- host-side helpers (capi.cu) ---------------------------------------
flsgpu_status set_error(flsgpu_status s, const char *fmt, ...);
flsgpu_status check_cuda(cudaError_t e, const char *what);
int sm_count();
void note_launch(uint64_t n = 1);

// Kernel grid: persistent, a whole number of waves over the SMs.
inline unsigned persistent_blocks(size_t work_warps, int warps_per_block,
                                  int blocks_per_sm) {
  const size_t need = (work_warps + warps_per_block - 1) / warps_per_block;
  const size_t cap = (size_t)sm_count() * (size_t)blocks_per_sm;
  size_t b = need < cap ? need : cap;
  return (unsigned)(b == 0 ? 1 : b);
}

// ---- device helpers ----------------------------------------------------
__device__ __forceinline__ uint32_t ld_stream_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ uint64_t ld_stream_u64(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.global.nc.L1::no_allocate.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ uint32_t funnel_r(uint32_t lo, uint32_t hi, uint32_t s) {
  return __funnelshift_r(lo, hi, s);
}

template <int W> __device__ __forceinline__ uint32_t mask32() {
  return W >= 32 ? 0xFFFFFFFFu : ((1u << (W & 31)) - 1u);
}
template <int W> __device__ __forceinline__ uint64_t mask64() {
  return W >= 64 ? ~0ull : ((1ull << (W & 63)) - 1ull);
}

template <int V> struct IntC { static constexpr int value = V; };

}  // namespace flsb200
