// autotune_table.h -- compiled defaults of the decode tuning.
//
// kPolicy32 / kPolicy64 (fixed at build time), per bit width of 32- / 64-bit
// lanes: bit 2 = streaming (evict-first) output stores, bit 16 = chunked
// decode of 64-bit half-lanes (two runs of 16 values), bit 64 = decode two
// same-width vectors per warp step.
//
// kPrefetch32 / kPrefetch64 and kVariant are the runtime defaults that the
// autotuner (flsgpu_b200.autotune, bench.py --workload autotune) measures on
// the device and replaces through flsgpu_tuning_set_*: per bit width, 1 =
// prefetch the next vector's packed lines into L2; per value type (u32, u64,
// f32, f64) and column kind (BP, FFOR, ALP, ALP extended), the kernel
// variant that FLSGPU_VARIANT_AUTO selects (1 = register-rich, 2 =
// register-capped for occupancy).  The values below are an autotuner result
// on B200 (tuning_header() in flsgpu_b200.py prints one in this form).
#pragma once

namespace flsb200 {
namespace tuned {
// 32-bit lanes: widths 0..32
constexpr unsigned char kPolicy32[33] = {
     0,  0,  0,  0,  0,  0,  0,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,
     2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2};
// 64-bit lanes: widths 0..64
constexpr unsigned char kPolicy64[65] = {
     0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,
     0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  2,
     2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,
     2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2,  2};
// runtime defaults (autotuner result)
constexpr unsigned char kPrefetch32[33] = {
     0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,
     0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0};
constexpr unsigned char kPrefetch64[65] = {
     0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  1,  1,
     1,  1,  1,  1,  1,  1,  1,  1,  1,  1,  1,  1,  1,  1,  1,  1,  1,
     1,  1,  1,  1,  1,  1,  1,  1,  0,  0,  0,  0,  0,  0,  0,  0,  0,
     0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0};
constexpr unsigned char kVariant[4][4] = {
    {1, 1, 1, 1}, {1, 1, 1, 1}, {1, 1, 1, 1}, {1, 1, 2, 2}};
}  // namespace tuned
}  // namespace flsb200
