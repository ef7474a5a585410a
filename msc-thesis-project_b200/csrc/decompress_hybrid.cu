// decompress_hybrid.cu -- decoding of hybrid columns, whose vectors are
// each ALP or ALP-RD (flsgpu_alphybrid_column).  The reference's
// alp::encode rejects data that calls for ALP-RD (encoder.hpp:208-211 picks
// the scheme per rowgroup, alp-bindings.cu throws EncodingException); a
// hybrid column keeps every vector in the scheme that suits it.
//
// One warp per vector over a persistent grid, as the single-scheme
// kernels: a vector's scheme byte selects the ALP decode (unpack, ALP
// transform, exception patch: store_one) or the ALP-RD decode (right and
// left parts staged in shared memory: rd_decode_vector); the branch is
// uniform across the warp.
#include "rd_decode.cuh"

namespace flsb200 {

// Each scheme's decode is a function of its own (not inlined), so that the
// two decoders' live ranges do not overlap in one loop body: inlined
// together they spilled 232 bytes per thread and decoded a half-ALP,
// half-ALP-RD column of 2^26 f64 values at 3224 GB/s, against 3781 GB/s
// this way (3616 with the ALP decode inlined).
template <typename T>
__device__ __noinline__ void hybrid_rd_vector(const RDParams &pr, size_t vi, int t,
                                              typename UintOf<T>::U *sr, uint16_t *sl) {
  using U = typename UintOf<T>::U;
  constexpr int MAXW = sizeof(U) * 8;
  const RDMeta m = rd_meta(pr, vi);
  if (m.rbw > MAXW || m.lbw > 16) {
    if (t == 0) flag_status(pr.d_status, FLSGPU_BAD_BIT_WIDTH);
    return;
  }
  rd_decode_vector<T>(pr, vi, m, t, sr, sl);
  __syncwarp();
}

template <typename T>
__device__ __noinline__ void hybrid_alp_vector(const KernelParams &pa, size_t vi, int t) {
  store_one<T, K_ALP, VAR_DEFAULT | VAR_OCC>(pa, vi, load_meta<T, K_ALP>(pa.c, vi, t), t);
}

template <typename T>
__global__ void __launch_bounds__(256, 2)
    k_hybrid(const __grid_constant__ KernelParams pa, const __grid_constant__ RDParams pr,
             const uint8_t *__restrict__ schemes) {
  using U = typename UintOf<T>::U;
  extern __shared__ __align__(16) unsigned char hy_smem[];
  U *sr = reinterpret_cast<U *>(hy_smem) + (threadIdx.x >> 5) * VEC;
  uint16_t *sl = reinterpret_cast<uint16_t *>(hy_smem + 8 * VEC * sizeof(U)) + (threadIdx.x >> 5) * VEC;
  const int t = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t vi = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; vi < pa.c.n_vecs;
       vi += nw) {
    const uint8_t sch = schemes[vi];
    if (sch == FLSGPU_SCHEME_ALP_RD) {
      hybrid_rd_vector<T>(pr, vi, t, sr, sl);
    } else if (sch == FLSGPU_SCHEME_ALP) {
      hybrid_alp_vector<T>(pa, vi, t);
    } else if (t == 0) {
      flag_status(pa.d_status, FLSGPU_BAD_PARAMETER_INDEX);
    }
  }
}

template <typename T>
static flsgpu_status decompress_hybrid(const flsgpu_alphybrid_column *c, T *d_out,
                                       const flsgpu_decode_opts *o, flsgpu_stream stream) {
  flsgpu_status s = check_opts(o);
  if (s) return s;
  if (!c) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column");
  KernelParams pa{};
  if ((s = fill(pa.c, &c->alp, o))) return s;
  RDParams pr{};
  if ((s = fill_rd(pr, &c->rd))) return s;
  pa.c.n_values = pr.n_values = c->n_values;
  pa.c.n_vecs = pr.n_vecs = vecs_of(c->n_values);
  if (pa.c.n_vecs == 0) return FLSGPU_OK;
  if (vecs_of(c->alp.n_values) != pa.c.n_vecs || vecs_of(c->rd.n_values) != pa.c.n_vecs)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "hybrid: sub-columns differ in length");
  if (!c->schemes) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "hybrid: null schemes");
  if (!d_out) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null output");
  if (((uintptr_t)d_out % sizeof(T)) != 0)
    return set_error(FLSGPU_ERR_MISALIGNED, "output not aligned");
  pa.d_status = pr.d_status = o ? o->d_status : nullptr;
  pa.out = pr.out = d_out;
  constexpr size_t smem = 8 * VEC * (sizeof(T) + sizeof(uint16_t));
  static int bps = 0;
  if (bps == 0) {
    cudaFuncSetAttribute(k_hybrid<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_hybrid<T>, 256, smem);
    bps = b > 0 ? b : 1;
  }
  const unsigned grid = persistent_blocks(pa.c.n_vecs, 8, bps);
  k_hybrid<T><<<grid, 256, smem, (cudaStream_t)stream>>>(pa, pr, c->schemes);
  note_launch();
  return check_cuda(cudaGetLastError(), "k_hybrid launch");
}

}  // namespace flsb200

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_decompress_alphybrid_f32(const flsgpu_alphybrid_column *c, float *o,
                                              const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress_hybrid<float>(c, o, op, s);
}

flsgpu_status flsgpu_decompress_alphybrid_f64(const flsgpu_alphybrid_column *c, double *o,
                                              const flsgpu_decode_opts *op, flsgpu_stream s) {
  return decompress_hybrid<double>(c, o, op, s);
}

}  // extern "C"
