// autotune_table.h -- per (type, bit width) unpacker policy of the decode
// kernels.  Bits: 1 = L2 prefetch of the next vector's packed lines,
// 2 = streaming (evict-first) output stores, 16 = chunked decode of 64-bit
// half-lanes (two runs of 16 values), 64 = decode two same-width vectors per
// warp step.  Chosen from the per-width variant
// sweep of the FFOR decode kernel on B200 (flsgpu_autotune / bench.py
// --workload autotune; numbers in profiles/ffor_decode_variants.md).
#pragma once

namespace flsb200 {
namespace tuned {
// 32-bit lanes: widths 0..32
constexpr unsigned char kPolicy32[33] = {
     0,  0,  0,  0,  0,  0,  0,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,
     3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3};
// 64-bit lanes: widths 0..64
constexpr unsigned char kPolicy64[65] = {
     0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,
     0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  3,
     3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,
     3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3,  3};
}  // namespace tuned
}  // namespace flsb200
