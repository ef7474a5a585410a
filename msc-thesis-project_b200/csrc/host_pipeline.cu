// host_pipeline.cu -- decoding columns that live in host memory into host
// memory, the way the reference's host bindings are used
// (bindings::decompress_column copies the column to the device, launches,
// synchronises and copies the values back: src/engine/kernels.cuh:94-112,
// src/generated-bindings/kernel-bindings.cuh:42-90), but pipelined: the
// column is cut into chunks of whole vectors, and per chunk the copy in
// (stream `in`), the decode (stream `comp`) and the copy out (stream `out`)
// run on their own streams over double-buffered device staging, so that the
// copies of neighbouring chunks in both directions overlap each other and
// the decode.  Host arrays should be pinned (page-locked) for the copies to
// be asynchronous and at full PCIe speed.
//
// A chunk's metadata arrays are copied as they are: vector offsets and
// exception offsets stay absolute, and the staged packed words and
// exceptions are addressed through a base pointer moved back by the chunk's
// first offset, so the decode kernels run unchanged on the chunk.
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "../../include/flsgpu_b200_ext.h"

struct flsgpu_host_pipeline {
  size_t chunk_vecs = 0;
  size_t seq = 0;  // chunks issued so far: slots alternate across calls
  cudaStream_t in = nullptr, comp = nullptr, out = nullptr;
  cudaEvent_t ev_in[2] = {}, ev_comp[2] = {}, ev_out[2] = {};
  // per slot: packed words, per-vector metadata, exceptions, output
  unsigned char *d_packed[2] = {}, *d_meta[2] = {}, *d_exc[2] = {}, *d_out[2] = {};
  void *d_tables = nullptr;  // factors / fractions when the column carries its own
};

namespace flsb200 {

// per-vector metadata bytes staged per chunk (all arrays, 8-byte aligned)
static size_t meta_bytes(size_t nv) { return 8 * nv * 5 + 64; }

// Copies [v0, v1) of a host column to slot `sl` and fills the device
// descriptor `dc` of that chunk (FFOR).
template <typename T>
static flsgpu_status stage_ffor(flsgpu_host_pipeline *p, int sl, const flsgpu_ffor_column *hc,
                                size_t v0, size_t v1, flsgpu_ffor_column &dc) {
  using U = typename UintOf<T>::U;
  constexpr size_t NL = 1024 / (sizeof(U) * 8);
  const size_t nv = v1 - v0;
  const size_t w0 = hc->bp.vector_offsets[v0];
  const size_t w1 = hc->bp.vector_offsets[v1 - 1] + (size_t)hc->bp.bit_widths[v1 - 1] * NL;
  if (w1 < w0 || w1 - w0 > p->chunk_vecs * 1024)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "host column: vector offsets out of order");
  // every vector's packed words must lie inside the staged range [w0, w1):
  // the decode addresses them through a base moved back by w0.  Widths
  // beyond the type are left to the kernel's metadata check (it skips the
  // vector and raises FLSGPU_BAD_BIT_WIDTH).
  for (size_t v = v0; v < v1; ++v) {
    const size_t bw = hc->bp.bit_widths[v], off = hc->bp.vector_offsets[v];
    if (bw > sizeof(U) * 8) continue;
    if (off < w0 || off > w1 || bw * NL > w1 - off)
      return set_error(FLSGPU_ERR_INVALID_ARGUMENT,
                       "host column: vector %zu packed words [%zu, +%zu) outside its chunk", v, off,
                       bw * NL);
  }
  unsigned char *m = p->d_meta[sl];
  size_t *d_offs = reinterpret_cast<size_t *>(m);
  U *d_bases = reinterpret_cast<U *>(m + 8 * nv);
  uint8_t *d_bw = m + 16 * nv;
  flsgpu_status st;
  const cudaStream_t s = p->in;
  if ((st = check_cuda(cudaMemcpyAsync(p->d_packed[sl], reinterpret_cast<const U *>(hc->bp.packed_array) + w0,
                                       (w1 - w0) * sizeof(U), cudaMemcpyHostToDevice, s), "copy in")) ||
      (st = check_cuda(cudaMemcpyAsync(d_offs, hc->bp.vector_offsets + v0, nv * sizeof(size_t),
                                       cudaMemcpyHostToDevice, s), "copy in")) ||
      (st = check_cuda(cudaMemcpyAsync(d_bw, hc->bp.bit_widths + v0, nv, cudaMemcpyHostToDevice, s),
                       "copy in")))
    return st;
  if (hc->bases &&
      (st = check_cuda(cudaMemcpyAsync(d_bases, reinterpret_cast<const U *>(hc->bases) + v0,
                                       nv * sizeof(U), cudaMemcpyHostToDevice, s), "copy in")))
    return st;
  dc = *hc;
  dc.bp.packed_array = reinterpret_cast<U *>(p->d_packed[sl]) - w0;
  dc.bp.bit_widths = d_bw;
  dc.bp.vector_offsets = d_offs;
  dc.bases = hc->bases ? d_bases : nullptr;
  return FLSGPU_OK;
}

template <typename T>
static flsgpu_status stage_alp(flsgpu_host_pipeline *p, int sl, const flsgpu_alp_column *hc,
                               size_t v0, size_t v1, flsgpu_alp_column &dc) {
  flsgpu_status st = stage_ffor<T>(p, sl, &hc->ffor, v0, v1, dc.ffor);
  if (st) return st;
  const size_t nv = v1 - v0;
  unsigned char *m = p->d_meta[sl];
  size_t *d_eoffs = reinterpret_cast<size_t *>(m + 24 * nv);
  uint16_t *d_counts = reinterpret_cast<uint16_t *>(m + 32 * nv);
  uint8_t *d_fac = m + 17 * nv, *d_frac = m + 18 * nv;
  const size_t e0 = hc->exceptions_offsets[v0];
  const size_t e1 = hc->exceptions_offsets[v1 - 1] + hc->counts[v1 - 1];
  if (e1 < e0 || e1 - e0 > p->chunk_vecs * 1024)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "host column: exception offsets out of order");
  for (size_t v = v0; v < v1; ++v) {
    const size_t eo = hc->exceptions_offsets[v], cnt = hc->counts[v];
    if (eo < e0 || eo > e1 || cnt > e1 - eo)
      return set_error(FLSGPU_ERR_INVALID_ARGUMENT,
                       "host column: vector %zu exceptions [%zu, +%zu) outside its chunk", v, eo, cnt);
  }
  unsigned char *ex = p->d_exc[sl];
  T *d_ex = reinterpret_cast<T *>(ex);
  uint16_t *d_pos = reinterpret_cast<uint16_t *>(ex + p->chunk_vecs * 1024 * sizeof(T));
  const cudaStream_t s = p->in;
  if ((st = check_cuda(cudaMemcpyAsync(d_fac, hc->factor_indices + v0, nv, cudaMemcpyHostToDevice, s), "copy in")) ||
      (st = check_cuda(cudaMemcpyAsync(d_frac, hc->fraction_indices + v0, nv, cudaMemcpyHostToDevice, s), "copy in")) ||
      (st = check_cuda(cudaMemcpyAsync(d_eoffs, hc->exceptions_offsets + v0, nv * sizeof(size_t),
                                       cudaMemcpyHostToDevice, s), "copy in")) ||
      (st = check_cuda(cudaMemcpyAsync(d_counts, hc->counts + v0, nv * sizeof(uint16_t),
                                       cudaMemcpyHostToDevice, s), "copy in")))
    return st;
  if (e1 > e0 &&
      ((st = check_cuda(cudaMemcpyAsync(d_ex, reinterpret_cast<const T *>(hc->exceptions) + e0,
                                        (e1 - e0) * sizeof(T), cudaMemcpyHostToDevice, s), "copy in")) ||
       (st = check_cuda(cudaMemcpyAsync(d_pos, hc->positions + e0, (e1 - e0) * sizeof(uint16_t),
                                        cudaMemcpyHostToDevice, s), "copy in"))))
    return st;
  dc.n_values = hc->n_values;
  dc.factors = hc->factors ? p->d_tables : nullptr;
  dc.fractions = hc->fractions ? reinterpret_cast<unsigned char *>(p->d_tables) + 256 : nullptr;
  dc.factor_indices = d_fac;
  dc.fraction_indices = d_frac;
  dc.n_exceptions = hc->n_exceptions;
  dc.exceptions_offsets = d_eoffs;
  dc.exceptions = d_ex - e0;
  dc.positions = d_pos - e0;
  dc.counts = d_counts;
  return FLSGPU_OK;
}

// A staged chunk is decoded through the library's own C entry points (the
// kernels are compiled once, in their translation units).
static flsgpu_status decode_chunk(const flsgpu_ffor_column *c, uint32_t *o,
                                  const flsgpu_decode_opts *op, flsgpu_stream s) {
  return flsgpu_decompress_ffor_u32(c, o, op, s);
}
static flsgpu_status decode_chunk(const flsgpu_ffor_column *c, uint64_t *o,
                                  const flsgpu_decode_opts *op, flsgpu_stream s) {
  return flsgpu_decompress_ffor_u64(c, o, op, s);
}
static flsgpu_status decode_chunk(const flsgpu_alp_column *c, float *o,
                                  const flsgpu_decode_opts *op, flsgpu_stream s) {
  return flsgpu_decompress_alp_f32(c, o, op, s);
}
static flsgpu_status decode_chunk(const flsgpu_alp_column *c, double *o,
                                  const flsgpu_decode_opts *op, flsgpu_stream s) {
  return flsgpu_decompress_alp_f64(c, o, op, s);
}

// The chunk loop: stage (stream in), decode (stream comp), copy out
// (stream out); slot reuse waits on the decode (inputs) and the copy out
// (output) of the chunk two before.
template <typename T, typename Col, typename Stage, typename Decode>
static flsgpu_status run_pipeline(flsgpu_host_pipeline *p, const Col *hc, size_t n_values,
                                  T *host_out, bool wait, Stage &&stage, Decode &&decode) {
  const size_t n_vecs = (n_values + 1023) / 1024;
  flsgpu_status st = FLSGPU_OK;
  for (size_t v0 = 0; v0 < n_vecs && !st; v0 += p->chunk_vecs) {
    const int sl = (int)(p->seq++ & 1);
    const size_t v1 = v0 + p->chunk_vecs < n_vecs ? v0 + p->chunk_vecs : n_vecs;
    if ((st = check_cuda(cudaStreamWaitEvent(p->in, p->ev_comp[sl], 0), "wait"))) break;
    Col dc;
    if ((st = stage(sl, v0, v1, dc))) break;
    if ((st = check_cuda(cudaEventRecord(p->ev_in[sl], p->in), "record")) ||
        (st = check_cuda(cudaStreamWaitEvent(p->comp, p->ev_in[sl], 0), "wait")) ||
        (st = check_cuda(cudaStreamWaitEvent(p->comp, p->ev_out[sl], 0), "wait")))
      break;
    // the chunk as a column of its own: values [v0 * 1024, v1 * 1024) of
    // the output, metadata indexed from v0
    const size_t n_chunk = (v1 * 1024 < n_values ? v1 * 1024 : n_values) - v0 * 1024;
    if ((st = decode(dc, n_chunk, reinterpret_cast<T *>(p->d_out[sl])))) break;
    if ((st = check_cuda(cudaEventRecord(p->ev_comp[sl], p->comp), "record")) ||
        (st = check_cuda(cudaStreamWaitEvent(p->out, p->ev_comp[sl], 0), "wait")) ||
        (st = check_cuda(cudaMemcpyAsync(host_out + v0 * 1024, p->d_out[sl], n_chunk * sizeof(T),
                                         cudaMemcpyDeviceToHost, p->out), "copy out")) ||
        (st = check_cuda(cudaEventRecord(p->ev_out[sl], p->out), "record")))
      break;
  }
  if (!wait && !st) return FLSGPU_OK;
  flsgpu_status ss = check_cuda(cudaStreamSynchronize(p->out), "sync");
  cudaStreamSynchronize(p->comp);
  cudaStreamSynchronize(p->in);
  return st ? st : ss;
}

// chunk metadata is indexed from the chunk's first vector: shift the
// descriptor's per-vector arrays so that index v0.. maps to 0..
template <typename T>
static flsgpu_status host_ffor(flsgpu_host_pipeline *p, const flsgpu_ffor_column *hc, T *host_out,
                               const flsgpu_decode_opts *o, bool wait) {
  if (!p || !hc || !host_out) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (!hc->bp.bit_widths || !hc->bp.vector_offsets || !hc->bp.packed_array)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null host array");
  return run_pipeline<T>(
      p, hc, hc->n_values, host_out, wait,
      [&](int sl, size_t v0, size_t v1, flsgpu_ffor_column &dc) {
        return stage_ffor<T>(p, sl, hc, v0, v1, dc);
      },
      [&](flsgpu_ffor_column &dc, size_t n, T *d_out) {
        dc.n_values = n;
        dc.bp.n_values = n;
        dc.bp.n_vecs = (n + 1023) / 1024;
        return decode_chunk(&dc, d_out, o, (flsgpu_stream)p->comp);
      });
}

template <typename T>
static flsgpu_status host_alp(flsgpu_host_pipeline *p, const flsgpu_alp_column *hc, T *host_out,
                              const flsgpu_decode_opts *o, bool wait) {
  if (!p || !hc || !host_out) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (!hc->ffor.bp.bit_widths || !hc->ffor.bp.vector_offsets || !hc->ffor.bp.packed_array ||
      !hc->ffor.bases || !hc->factor_indices || !hc->fraction_indices ||
      !hc->exceptions_offsets || !hc->counts)
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null host array");
  constexpr bool F64 = sizeof(T) == 8;
  if (!wait && (hc->factors || hc->fractions))
    return set_error(FLSGPU_ERR_UNSUPPORTED,
                     "asynchronous host decode needs the built-in factor / fraction tables");
  if (hc->factors || hc->fractions) {
    flsgpu_status st = FLSGPU_OK;
    if (hc->factors)
      st = check_cuda(cudaMemcpyAsync(p->d_tables, hc->factors, (F64 ? 19 : 10) * sizeof(T),
                                      cudaMemcpyHostToDevice, p->in), "copy tables");
    if (!st && hc->fractions)
      st = check_cuda(cudaMemcpyAsync(reinterpret_cast<unsigned char *>(p->d_tables) + 256,
                                      hc->fractions, (F64 ? 21 : 11) * sizeof(T),
                                      cudaMemcpyHostToDevice, p->in), "copy tables");
    if (st) return st;
  }
  return run_pipeline<T>(
      p, hc, hc->n_values, host_out, wait,
      [&](int sl, size_t v0, size_t v1, flsgpu_alp_column &dc) {
        return stage_alp<T>(p, sl, hc, v0, v1, dc);
      },
      [&](flsgpu_alp_column &dc, size_t n, T *d_out) {
        dc.n_values = n;
        dc.ffor.n_values = n;
        dc.ffor.bp.n_values = n;
        dc.ffor.bp.n_vecs = (n + 1023) / 1024;
        return decode_chunk(&dc, d_out, o, (flsgpu_stream)p->comp);
      });
}

}  // namespace flsb200

using namespace flsb200;

extern "C" {

void flsgpu_host_pipeline_destroy(flsgpu_host_pipeline *p) {
  if (!p) return;
  if (p->in) cudaStreamSynchronize(p->in);
  if (p->comp) cudaStreamSynchronize(p->comp);
  if (p->out) cudaStreamSynchronize(p->out);
  for (int i = 0; i < 2; ++i) {
    cudaFree(p->d_packed[i]);
    cudaFree(p->d_meta[i]);
    cudaFree(p->d_exc[i]);
    cudaFree(p->d_out[i]);
    if (p->ev_in[i]) cudaEventDestroy(p->ev_in[i]);
    if (p->ev_comp[i]) cudaEventDestroy(p->ev_comp[i]);
    if (p->ev_out[i]) cudaEventDestroy(p->ev_out[i]);
  }
  cudaFree(p->d_tables);
  if (p->in) cudaStreamDestroy(p->in);
  if (p->comp) cudaStreamDestroy(p->comp);
  if (p->out) cudaStreamDestroy(p->out);
  delete p;
}

flsgpu_status flsgpu_host_pipeline_create(size_t chunk_values, flsgpu_host_pipeline **out) {
  if (!out || chunk_values < 1024 || (chunk_values % 1024))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "chunk_values must be a positive multiple of 1024");
  auto *p = new flsgpu_host_pipeline();
  p->chunk_vecs = chunk_values / 1024;
  const size_t nv = p->chunk_vecs;
  flsgpu_status st = FLSGPU_OK;
  for (cudaStream_t *s : {&p->in, &p->comp, &p->out})
    if (!st) st = check_cuda(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking), "stream");
  for (int i = 0; i < 2 && !st; ++i) {
    st = check_cuda(cudaEventCreateWithFlags(&p->ev_in[i], cudaEventDisableTiming), "event");
    if (!st) st = check_cuda(cudaEventCreateWithFlags(&p->ev_comp[i], cudaEventDisableTiming), "event");
    if (!st) st = check_cuda(cudaEventCreateWithFlags(&p->ev_out[i], cudaEventDisableTiming), "event");
    if (!st) st = check_cuda(cudaMalloc(&p->d_packed[i], nv * 1024 * 8), "cudaMalloc staging");
    if (!st) st = check_cuda(cudaMalloc(&p->d_meta[i], meta_bytes(nv)), "cudaMalloc staging");
    if (!st) st = check_cuda(cudaMalloc(&p->d_exc[i], nv * 1024 * (8 + 2)), "cudaMalloc staging");
    if (!st) st = check_cuda(cudaMalloc(&p->d_out[i], nv * 1024 * 8), "cudaMalloc staging");
  }
  if (!st) st = check_cuda(cudaMalloc(&p->d_tables, 512), "cudaMalloc tables");
  if (st) {
    flsgpu_host_pipeline_destroy(p);
    return st;
  }
  *out = p;
  return FLSGPU_OK;
}

flsgpu_status flsgpu_host_decompress_ffor_u32(flsgpu_host_pipeline *p, const flsgpu_ffor_column *c,
                                              uint32_t *host_out, const flsgpu_decode_opts *o) {
  return host_ffor<uint32_t>(p, c, host_out, o, true);
}
flsgpu_status flsgpu_host_decompress_ffor_u64(flsgpu_host_pipeline *p, const flsgpu_ffor_column *c,
                                              uint64_t *host_out, const flsgpu_decode_opts *o) {
  return host_ffor<uint64_t>(p, c, host_out, o, true);
}
flsgpu_status flsgpu_host_decompress_alp_f32(flsgpu_host_pipeline *p, const flsgpu_alp_column *c,
                                             float *host_out, const flsgpu_decode_opts *o) {
  return host_alp<float>(p, c, host_out, o, true);
}
flsgpu_status flsgpu_host_decompress_alp_f64(flsgpu_host_pipeline *p, const flsgpu_alp_column *c,
                                             double *host_out, const flsgpu_decode_opts *o) {
  return host_alp<double>(p, c, host_out, o, true);
}
flsgpu_status flsgpu_host_decompress_ffor_u32_async(flsgpu_host_pipeline *p,
                                                    const flsgpu_ffor_column *c, uint32_t *host_out,
                                                    const flsgpu_decode_opts *o) {
  return host_ffor<uint32_t>(p, c, host_out, o, false);
}
flsgpu_status flsgpu_host_decompress_ffor_u64_async(flsgpu_host_pipeline *p,
                                                    const flsgpu_ffor_column *c, uint64_t *host_out,
                                                    const flsgpu_decode_opts *o) {
  return host_ffor<uint64_t>(p, c, host_out, o, false);
}
flsgpu_status flsgpu_host_decompress_alp_f32_async(flsgpu_host_pipeline *p,
                                                   const flsgpu_alp_column *c, float *host_out,
                                                   const flsgpu_decode_opts *o) {
  return host_alp<float>(p, c, host_out, o, false);
}
flsgpu_status flsgpu_host_decompress_alp_f64_async(flsgpu_host_pipeline *p,
                                                   const flsgpu_alp_column *c, double *host_out,
                                                   const flsgpu_decode_opts *o) {
  return host_alp<double>(p, c, host_out, o, false);
}
flsgpu_status flsgpu_host_pipeline_sync(flsgpu_host_pipeline *p) {
  if (!p) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null pipeline");
  flsgpu_status st = check_cuda(cudaStreamSynchronize(p->out), "sync");
  cudaStreamSynchronize(p->comp);
  cudaStreamSynchronize(p->in);
  return st;
}

}  // extern "C"
