// batch.cu -- host side of the batched persistent decode of many columns of
// uneven length, type and bit width, replayable from a captured CUDA graph.
//
// The reference launches one kernel per column and synchronises after each
// (src/engine/kernels.cuh:94-112, multi-column-host-kernels.cuh:32-115).
// Here the columns are grouped by value type; per group a device table
// describes every column and the vectors of all its columns form one index
// space (prefix sums of the per-column vector counts), which a persistent
// grid of warps consumes in chunks from an atomic counter (batch.cuh), so
// short and long columns load-balance and a batch costs one launch per value
// type and float kind present (at most six).  Per vector the warp dispatches on the
// column's encoding and the vector's bit width to the same per-width
// unpackers and autotuned policies as the single-column kernels.
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "batch.cuh"
#include "../../include/flsgpu_b200_ext.h"

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// Columns are grouped by value type; each group has its own descriptor
// table, prefix array and work counter in one device allocation each.
struct flsgpu_batch {
  std::vector<flsb200::BatchEntry> host_table;    // grouped by type
  std::vector<size_t> host_prefix;                // per group, n + 1 entries each
  std::vector<flsgpu_batch_column> cols;          // for the per-column path
  // group g = 2 * value type + (ALP extended ? 1 : 0)
  int group_cols[8] = {};
  size_t group_first[8] = {};                     // first entry of each group
  size_t group_prefix_at[8] = {};                 // first prefix slot of each group
  size_t group_vecs[8] = {};
  flsb200::BatchEntry *d_table = nullptr;
  size_t *d_prefix = nullptr;
  unsigned long long *d_counter = nullptr;        // one per group (8)
  int n_cols = 0;
  size_t total_vecs = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // fork / join of the per-type launches: they run concurrently, so one
  // group's tail overlaps the next group's start
  cudaStream_t side[7] = {};
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev_join[7] = {};
  flsgpu_decode_opts opts{};
  bool has_opts = false;
};

namespace flsb200 {

static flsgpu_status fill_entry(BatchEntry &e, const flsgpu_batch_column &bc,
                                const flsgpu_decode_opts *o) {
  e = BatchEntry{};
  flsgpu_status s;
  int kind;
  switch (bc.encoding) {
    case FLSGPU_ENCODING_BP:
      s = fill(e.p.c, static_cast<const flsgpu_bp_column *>(bc.column), o);
      kind = K_BP;
      break;
    case FLSGPU_ENCODING_FFOR:
      s = fill(e.p.c, static_cast<const flsgpu_ffor_column *>(bc.column), o);
      kind = K_FFOR;
      break;
    case FLSGPU_ENCODING_ALP:
      s = fill(e.p.c, static_cast<const flsgpu_alp_column *>(bc.column), o);
      kind = K_ALP;
      break;
    case FLSGPU_ENCODING_ALP_EXTENDED:
      s = fill(e.p.c, static_cast<const flsgpu_alpx_column *>(bc.column), o);
      kind = K_ALPX;
      break;
    default:
      return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "unknown encoding %u", bc.encoding);
  }
  if (s) return s;
  const bool is_float = bc.type == FLSGPU_TYPE_F32 || bc.type == FLSGPU_TYPE_F64;
  const bool is_alp = kind == K_ALP || kind == K_ALPX;
  if (bc.type > FLSGPU_TYPE_F64 || is_float != is_alp)
    return set_error(FLSGPU_ERR_UNSUPPORTED, "type %u with encoding %u", bc.type, bc.encoding);
  if (e.p.c.n_vecs && !bc.d_out) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null output");
  e.p.out = bc.d_out;
  e.p.d_status = o ? o->d_status : nullptr;
  e.kind = (uint32_t)kind;
  return FLSGPU_OK;
}

static flsgpu_status launch_batch(flsgpu_batch *b, cudaStream_t s) {
  using L = flsgpu_status (*)(const BatchEntry *, const size_t *, int, size_t,
                              unsigned long long *, cudaStream_t, int);
  static const L launch[4] = {launch_batch_u32, launch_batch_u64, launch_batch_f32,
                              launch_batch_f64};
  int groups[8], n = 0;
  for (int g = 0; g < 8; ++g)
    if (b->group_vecs[g] != 0) groups[n++] = g;
  flsgpu_status st;
  if (n > 1 && (st = check_cuda(cudaEventRecord(b->ev_fork, s), "fork"))) return st;
  for (int i = 0; i < n; ++i) {
    const int g = groups[i];
    cudaStream_t gs = i == 0 ? s : b->side[i - 1];
    if (i > 0 && (st = check_cuda(cudaStreamWaitEvent(gs, b->ev_fork, 0), "fork wait"))) return st;
    if ((st = launch[g >> 1](b->d_table + b->group_first[g], b->d_prefix + b->group_prefix_at[g],
                             b->group_cols[g], b->group_vecs[g], b->d_counter + g, gs, g & 1)))
      return st;
    if (i > 0 && ((st = check_cuda(cudaEventRecord(b->ev_join[i - 1], gs), "join")) ||
                  (st = check_cuda(cudaStreamWaitEvent(s, b->ev_join[i - 1], 0), "join wait"))))
      return st;
  }
  return FLSGPU_OK;
}

}  // namespace flsb200

using namespace flsb200;

extern "C" {

flsgpu_status flsgpu_batch_create(const flsgpu_batch_column *columns, size_t n_columns,
                                  const flsgpu_decode_opts *opts, flsgpu_batch **out) {
  if (!out || (n_columns && !columns))
    return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null batch arguments");
  flsgpu_status s = check_opts(opts);
  if (s) return s;
  if (n_columns > (1u << 30)) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "too many columns");
  auto *b = new flsgpu_batch();
  b->n_cols = (int)n_columns;
  b->cols.assign(columns, columns + n_columns);
  if (opts) {
    b->opts = *opts;
    b->has_opts = true;
  }
  std::vector<BatchEntry> entries(n_columns);
  for (size_t i = 0; i < n_columns; ++i) {
    if (!columns[i].column) {
      delete b;
      return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null column %zu", i);
    }
    if ((s = fill_entry(entries[i], columns[i], opts))) {
      delete b;
      return s;
    }
  }
  // group by type: table entries in group order, one prefix array per group
  for (int g = 0; g < 8; ++g) {
    b->group_first[g] = b->host_table.size();
    b->group_prefix_at[g] = b->host_prefix.size();
    b->host_prefix.push_back(0);
    for (size_t i = 0; i < n_columns; ++i) {
      const int gi = 2 * (int)columns[i].type +
                     (columns[i].encoding == FLSGPU_ENCODING_ALP_EXTENDED ? 1 : 0);
      if (gi != g) continue;
      b->host_table.push_back(entries[i]);
      b->host_prefix.push_back(b->host_prefix.back() + entries[i].p.c.n_vecs);
      b->group_cols[g]++;
    }
    b->group_vecs[g] = b->host_prefix.back();
    b->total_vecs += b->group_vecs[g];
  }
  const size_t tb = sizeof(BatchEntry) * (b->host_table.size() ? b->host_table.size() : 1);
  for (int i = 0; i < 7 && !s; ++i)
    s = check_cuda(cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking), "stream");
  for (int i = 0; i < 7 && !s; ++i)
    s = check_cuda(cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming), "event");
  if (!s) s = check_cuda(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming), "event");
  if (s) {
    flsgpu_batch_destroy(b);
    return s;
  }
  if ((s = check_cuda(cudaMalloc(&b->d_table, tb), "cudaMalloc table")) ||
      (s = check_cuda(cudaMalloc(&b->d_prefix, sizeof(size_t) * b->host_prefix.size()), "cudaMalloc prefix")) ||
      (s = check_cuda(cudaMalloc(&b->d_counter, 8 * sizeof(unsigned long long)), "cudaMalloc counter"))) {
    flsgpu_batch_destroy(b);
    return s;
  }
  if (!b->host_table.empty())
    s = check_cuda(cudaMemcpy(b->d_table, b->host_table.data(), tb, cudaMemcpyHostToDevice), "copy");
  if (!s)
    s = check_cuda(cudaMemcpy(b->d_prefix, b->host_prefix.data(), sizeof(size_t) * b->host_prefix.size(),
                              cudaMemcpyHostToDevice), "copy");
  if (s) {
    flsgpu_batch_destroy(b);
    return s;
  }
  *out = b;
  return FLSGPU_OK;
}

flsgpu_status flsgpu_batch_decompress(flsgpu_batch *b, flsgpu_stream stream) {
  if (!b) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null batch");
  if (b->total_vecs == 0) return FLSGPU_OK;
  return launch_batch(b, (cudaStream_t)stream);
}

flsgpu_status flsgpu_batch_capture_graph(flsgpu_batch *b, flsgpu_stream stream) {
  if (!b) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null batch");
  cudaStream_t s = (cudaStream_t)stream;
  bool own = false;
  if (!s) {
    flsgpu_status st = check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    if (st) return st;
    own = true;
  }
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  flsgpu_status st = check_cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture");
  if (!st) {
    flsgpu_status ls = b->total_vecs ? launch_batch(b, s) : FLSGPU_OK;
    flsgpu_status es = check_cuda(cudaStreamEndCapture(s, &b->graph), "end capture");
    st = ls ? ls : es;
  }
  if (!st) st = check_cuda(cudaGraphInstantiate(&b->exec, b->graph, 0), "instantiate");
  if (own) cudaStreamDestroy(s);
  return st;
}

flsgpu_status flsgpu_batch_replay(flsgpu_batch *b, flsgpu_stream stream) {
  if (!b || !b->exec) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "no captured graph");
  flsgpu_status st = check_cuda(cudaGraphLaunch(b->exec, (cudaStream_t)stream), "graph launch");
  if (!st) note_launch();
  return st;
}

flsgpu_status flsgpu_batch_decompress_each(flsgpu_batch *b, int sync_each, flsgpu_stream stream) {
  if (!b) return set_error(FLSGPU_ERR_INVALID_ARGUMENT, "null batch");
  const flsgpu_decode_opts *o = b->has_opts ? &b->opts : nullptr;
  for (const auto &c : b->cols) {
    flsgpu_status s = FLSGPU_ERR_UNSUPPORTED;
    const int key = (int)(c.type * 4 + c.encoding);
    switch (key) {
      case FLSGPU_TYPE_U32 * 4 + FLSGPU_ENCODING_BP:
        s = flsgpu_decompress_bp_u32((const flsgpu_bp_column *)c.column, (uint32_t *)c.d_out, o, stream);
        break;
      case FLSGPU_TYPE_U64 * 4 + FLSGPU_ENCODING_BP:
        s = flsgpu_decompress_bp_u64((const flsgpu_bp_column *)c.column, (uint64_t *)c.d_out, o, stream);
        break;
      case FLSGPU_TYPE_U32 * 4 + FLSGPU_ENCODING_FFOR:
        s = flsgpu_decompress_ffor_u32((const flsgpu_ffor_column *)c.column, (uint32_t *)c.d_out, o, stream);
        break;
      case FLSGPU_TYPE_U64 * 4 + FLSGPU_ENCODING_FFOR:
        s = flsgpu_decompress_ffor_u64((const flsgpu_ffor_column *)c.column, (uint64_t *)c.d_out, o, stream);
        break;
      case FLSGPU_TYPE_F32 * 4 + FLSGPU_ENCODING_ALP:
        s = flsgpu_decompress_alp_f32((const flsgpu_alp_column *)c.column, (float *)c.d_out, o, stream);
        break;
      case FLSGPU_TYPE_F64 * 4 + FLSGPU_ENCODING_ALP:
        s = flsgpu_decompress_alp_f64((const flsgpu_alp_column *)c.column, (double *)c.d_out, o, stream);
        break;
      case FLSGPU_TYPE_F32 * 4 + FLSGPU_ENCODING_ALP_EXTENDED:
        s = flsgpu_decompress_alpx_f32((const flsgpu_alpx_column *)c.column, (float *)c.d_out, o, stream);
        break;
      case FLSGPU_TYPE_F64 * 4 + FLSGPU_ENCODING_ALP_EXTENDED:
        s = flsgpu_decompress_alpx_f64((const flsgpu_alpx_column *)c.column, (double *)c.d_out, o, stream);
        break;
      default:
        return set_error(FLSGPU_ERR_UNSUPPORTED, "type %u encoding %u", c.type, c.encoding);
    }
    if (s) return s;
    if (sync_each && (s = check_cuda(cudaStreamSynchronize((cudaStream_t)stream), "sync")))
      return s;
  }
  return FLSGPU_OK;
}

size_t flsgpu_batch_total_vectors(const flsgpu_batch *b) { return b ? b->total_vecs : 0; }

void flsgpu_batch_destroy(flsgpu_batch *b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->d_table) cudaFree(b->d_table);
  if (b->d_prefix) cudaFree(b->d_prefix);
  if (b->d_counter) cudaFree(b->d_counter);
  for (int i = 0; i < 7; ++i) {
    if (b->side[i]) cudaStreamDestroy(b->side[i]);
    if (b->ev_join[i]) cudaEventDestroy(b->ev_join[i]);
  }
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  delete b;
}

}  // extern "C"
