// extended.cu -- conversion of an ALP column's exceptions into the
// lane-divided layout of ALPExtendedColumn on the GPU (the reference does it
// on the host: host::ALPColumn::convert_exceptions_to_lane_divided_format /
// create_extended_column, src/flsgpu/structs.cuh:231-308).
//
// Per vector (one warp): the vector's exceptions are regrouped by FastLanes
// lane (position % N_LANES), keeping their order within a lane, and each
// lane gets offsets_counts[v * N_LANES + lane] = (count << 10) | (offset of
// the lane's first exception within the vector), stored as 16 bits: like the
// reference, a 64-bit lane with 64 exceptions wraps its 6-bit count.  The
// vectors keep their exception offsets, so exceptions_offsets is shared with
// the source column.
//
// Two passes over the vector's list: lane counts (shared-memory counters),
// their exclusive prefix, then a stable placement in rounds of 32: a
// thread's slot is its lane's base, plus the exceptions of the lane placed in
// earlier rounds, plus those before it in this round (__match_any_sync).
#include "kernels.cuh"

namespace flsb200 {

template <typename T>
__global__ void __launch_bounds__(256) k_to_extended(const flsgpu_alp_column c, size_t n_vecs,
                                                     T *out_exc, uint16_t *out_pos,
                                                     uint16_t *out_oc) {
  using U = typename UintOf<T>::U;
  constexpr int NL = Lanes<U>::N;
  __shared__ uint32_t s_cnt[8][32], s_run[8][32];
  const int t = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t *cnt = s_cnt[wib], *run = s_run[wib];
  const T *exc = reinterpret_cast<const T *>(c.exceptions);
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t v = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n_vecs; v += nw) {
    const uint32_t count = c.counts[v];
    const size_t eo = c.exceptions_offsets[v];
    __syncwarp();
    cnt[t] = 0;
    run[t] = 0;
    __syncwarp();
    for (uint32_t i = t; i < count; i += 32) atomicAdd(&cnt[c.positions[eo + i] % NL], 1u);
    __syncwarp();
    // exclusive prefix of the lane counts
    const uint32_t mine = t < NL ? cnt[t] : 0u;
    uint32_t incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (t >= o) incl += y;
    }
    const uint32_t base_t = incl - mine;
    if (t < NL) out_oc[v * NL + t] = (uint16_t)((mine << 10) | base_t);
    // stable placement, 32 exceptions per round
    for (uint32_t r = 0; r < count; r += 32) {
      const uint32_t i = r + t;
      const bool act = i < count;
      const uint32_t p = act ? c.positions[eo + i] : 0u;
      const int key = act ? (int)(p % NL) : 32 + t;  // inactive threads match only themselves
      const unsigned grp = __match_any_sync(0xffffffffu, key);
      const uint32_t rank = __popc(grp & ((1u << t) - 1u));
      const uint32_t lane_base = __shfl_sync(0xffffffffu, base_t, key & 31);
      if (act) {
        const uint32_t slot = lane_base + run[key] + rank;
        out_exc[eo + slot] = exc[eo + i];
        out_pos[eo + slot] = (uint16_t)p;
      }
      __syncwarp();
      if (act && rank == 0) run[key] += __popc(grp);
      __syncwarp();
    }
  }
}

template <typename T>
static flsgpu_status to_extended(const flsgpu_alp_column *src, T *d_exc, uint16_t *d_pos,
                                 uint16_t *d_oc, flsgpu_alpx_column *dst, flsgpu_stream stream) {
  if (!src || !dst) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  const size_t n_vecs = vecs_of(src->n_values);
  if (n_vecs && (!src->counts || !src->exceptions_offsets || !d_oc))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null counts / offsets / output");
  if (src->n_exceptions && (!src->exceptions || !src->positions || !d_exc || !d_pos))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null exception arrays");
  if (n_vecs) {
    const unsigned grid = persistent_blocks(n_vecs, 8, 8);
    k_to_extended<T><<<grid, 256, 0, (cudaStream_t)stream>>>(*src, n_vecs, d_exc, d_pos, d_oc);
    note_launch();
    flsgpu_status s = check_cuda(cudaGetLastError(), "k_to_extended launch");
    if (s) return s;
  }
  dst->n_values = src->n_values;
  dst->ffor = src->ffor;
  dst->factors = src->factors;
  dst->fractions = src->fractions;
  dst->factor_indices = src->factor_indices;
  dst->fraction_indices = src->fraction_indices;
  dst->n_exceptions = src->n_exceptions;
  dst->exceptions_offsets = src->exceptions_offsets;
  dst->exceptions = d_exc;
  dst->positions = d_pos;
  dst->offsets_counts = d_oc;
  return FLSGPU_OK;
}

}  // namespace flsb200

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_alp_to_extended_f32(const flsgpu_alp_column *src, float *d_exceptions,
                                         uint16_t *d_positions, uint16_t *d_offsets_counts,
                                         flsgpu_alpx_column *dst, flsgpu_stream stream) {
  return to_extended<float>(src, d_exceptions, d_positions, d_offsets_counts, dst, stream);
}

flsgpu_status flsgpu_alp_to_extended_f64(const flsgpu_alp_column *src, double *d_exceptions,
                                         uint16_t *d_positions, uint16_t *d_offsets_counts,
                                         flsgpu_alpx_column *dst, flsgpu_stream stream) {
  return to_extended<double>(src, d_exceptions, d_positions, d_offsets_counts, dst, stream);
}

}  // extern "C"
