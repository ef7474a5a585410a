/*
 * flsgpu_b200_ext.h -- C ABI of the parts of libflsgpu_b200.so that have no
 * counterpart in the reference: batched persistent decode of many columns,
 * the fused pair query over compressed columns, and the GPU ALP encoder
 * with its learned (exponent, factor) proposal network.
 * Conventions as in flsgpu_b200.h.
 */
#ifndef FLSGPU_B200_EXT_H
#define FLSGPU_B200_EXT_H

#include "flsgpu_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- batched persistent decode (no reference counterpart; replaces one
 *      launch + cudaDeviceSynchronize per column, src/engine/kernels.cuh:
 *      94-112) -------------------------------------------------------------
 * Columns are grouped by value type; within a group all vectors of all
 * columns form one index space that a persistent grid takes in chunks from
 * an atomic counter, so a batch of columns of uneven length, type and bit
 * width decodes in one launch per value type present (ALP and ALP-extended
 * float columns in separate launches; at most six).  The
 * decode per vector is the single-column kernels' (same per-width autotuned
 * unpackers). */
typedef enum flsgpu_type {
  FLSGPU_TYPE_U32 = 0, FLSGPU_TYPE_U64 = 1, FLSGPU_TYPE_F32 = 2, FLSGPU_TYPE_F64 = 3
} flsgpu_type;
typedef enum flsgpu_encoding {
  FLSGPU_ENCODING_BP = 0, FLSGPU_ENCODING_FFOR = 1, FLSGPU_ENCODING_ALP = 2,
  FLSGPU_ENCODING_ALP_EXTENDED = 3
} flsgpu_encoding;
typedef struct flsgpu_batch_column {
  uint32_t type;       /* flsgpu_type */
  uint32_t encoding;   /* flsgpu_encoding; floats need ALP, integers BP/FFOR */
  const void *column;  /* host pointer to the matching flsgpu_*_column */
  void *d_out;         /* device output, column n_values elements */
} flsgpu_batch_column;
typedef struct flsgpu_batch flsgpu_batch;

/* Copies the descriptors into a device table (allocates ~200 B per column).
 * The descriptors' device arrays must outlive the batch. */
flsgpu_status flsgpu_batch_create(const flsgpu_batch_column *columns, size_t n_columns,
                                  const flsgpu_decode_opts *opts, flsgpu_batch **out);
/* One persistent launch per group (plus counter resets); the groups'
 * launches are forked onto the batch's own streams and joined back into
 * `stream`, so they may run concurrently. */
flsgpu_status flsgpu_batch_decompress(flsgpu_batch *batch, flsgpu_stream stream);
/* Captures flsgpu_batch_decompress into a CUDA graph held by the batch
 * (NULL stream: a private stream is used); flsgpu_batch_replay launches it. */
flsgpu_status flsgpu_batch_capture_graph(flsgpu_batch *batch, flsgpu_stream stream);
flsgpu_status flsgpu_batch_replay(flsgpu_batch *batch, flsgpu_stream stream);
/* The comparison path: one flsgpu_decompress_* launch per column; with
 * sync_each the stream is synchronised after every launch, as the
 * reference's host launchers do (src/engine/kernels.cuh:106). */
flsgpu_status flsgpu_batch_decompress_each(flsgpu_batch *batch, int sync_each,
                                           flsgpu_stream stream);
size_t flsgpu_batch_total_vectors(const flsgpu_batch *batch);
void flsgpu_batch_destroy(flsgpu_batch *batch);

/* ---- decode tuning (no reference counterpart; the reference fixes its
 *      unpacker per build in the generated bindings) ----------------------
 * Process-wide state read at every launch: the kernel variant that
 * FLSGPU_VARIANT_AUTO selects per value type (0 u32, 1 u64, 2 f32, 3 f64)
 * and column kind (0 BP, 1 FFOR, 2 ALP, 3 ALP extended), and per lane width
 * (32 or 64) a bit mask over bit widths 0..127: bit w asks the decode to
 * prefetch the next vector's packed lines into L2 when that vector has
 * width w.  Defaults are compiled in (autotune_table.h); the autotuner
 * (flsgpu_b200.autotune) measures the variants on the device and installs
 * its choice here.  Not synchronised with launches in flight: set it before
 * decoding. */
flsgpu_status flsgpu_tuning_set_variant(uint32_t type, uint32_t kind, uint32_t variant);
flsgpu_status flsgpu_tuning_get_variant(uint32_t type, uint32_t kind, uint32_t *variant);
flsgpu_status flsgpu_tuning_set_prefetch(uint32_t lane_bits, const uint64_t mask[2]);
flsgpu_status flsgpu_tuning_get_prefetch(uint32_t lane_bits, uint64_t mask[2]);

/* ---- decode of host-resident columns, pipelined (the reference's host
 *      binding copies a whole column in, decodes, synchronises and copies
 *      back: src/engine/kernels.cuh:94-112) ---------------------------------
 * The column descriptor holds HOST pointers (pin them for asynchronous,
 * full-speed copies); the decoded values land in host_out.  Chunks of
 * chunk_values values (a multiple of 1024) are copied in, decoded and
 * copied out on three streams over double-buffered device staging that the
 * pipeline allocates once (about 34 bytes per chunk value per slot), so
 * copies in both directions overlap the decode.  factors / fractions may
 * be host tables or NULL.  Each call returns when host_out is complete;
 * calls on one pipeline must not overlap. */
typedef struct flsgpu_host_pipeline flsgpu_host_pipeline;
flsgpu_status flsgpu_host_pipeline_create(size_t chunk_values, flsgpu_host_pipeline **out);
void flsgpu_host_pipeline_destroy(flsgpu_host_pipeline *pipeline);
flsgpu_status flsgpu_host_decompress_ffor_u32(flsgpu_host_pipeline *pipeline,
                                              const flsgpu_ffor_column *host_column,
                                              uint32_t *host_out, const flsgpu_decode_opts *opts);
flsgpu_status flsgpu_host_decompress_ffor_u64(flsgpu_host_pipeline *pipeline,
                                              const flsgpu_ffor_column *host_column,
                                              uint64_t *host_out, const flsgpu_decode_opts *opts);
flsgpu_status flsgpu_host_decompress_alp_f32(flsgpu_host_pipeline *pipeline,
                                             const flsgpu_alp_column *host_column,
                                             float *host_out, const flsgpu_decode_opts *opts);
flsgpu_status flsgpu_host_decompress_alp_f64(flsgpu_host_pipeline *pipeline,
                                             const flsgpu_alp_column *host_column,
                                             double *host_out, const flsgpu_decode_opts *opts);
/* The same without waiting: the chunks join the pipeline's queue behind
 * those of earlier calls (the slots alternate across calls), so a series of
 * columns streams without draining between them.  The host arrays and
 * host_out of every call must stay valid and untouched until
 * flsgpu_host_pipeline_sync returns; the outputs are complete only then.
 * Columns must use the built-in factor / fraction tables. */
flsgpu_status flsgpu_host_decompress_ffor_u32_async(flsgpu_host_pipeline *pipeline,
                                                    const flsgpu_ffor_column *host_column,
                                                    uint32_t *host_out,
                                                    const flsgpu_decode_opts *opts);
flsgpu_status flsgpu_host_decompress_ffor_u64_async(flsgpu_host_pipeline *pipeline,
                                                    const flsgpu_ffor_column *host_column,
                                                    uint64_t *host_out,
                                                    const flsgpu_decode_opts *opts);
flsgpu_status flsgpu_host_decompress_alp_f32_async(flsgpu_host_pipeline *pipeline,
                                                   const flsgpu_alp_column *host_column,
                                                   float *host_out, const flsgpu_decode_opts *opts);
flsgpu_status flsgpu_host_decompress_alp_f64_async(flsgpu_host_pipeline *pipeline,
                                                   const flsgpu_alp_column *host_column,
                                                   double *host_out, const flsgpu_decode_opts *opts);
flsgpu_status flsgpu_host_pipeline_sync(flsgpu_host_pipeline *pipeline);

/* ---- fused pair query over compressed columns (no reference counterpart)
 * For each pair i: d_results[i] = sum of A_i[k] over positions k with
 * B_i[k] < median(B_i), where A_i is an f64 ALP column, B_i a u32 FFOR
 * column of the same n_values, and median(B_i) the element of rank
 * floor((n-1)/2) of B_i's values (radix select, four 8-bit passes over the
 * packed B).  The sum follows the fixed reduction tree of flsgpu_sum_alp_f64
 * restricted to the selected positions, so results are reproducible bit
 * for bit.  d_medians (optional) receives each median.  At most 2^21
 * vectors per pair. */
typedef struct flsgpu_pair_query flsgpu_pair_query;
flsgpu_status flsgpu_pair_query_create(const flsgpu_alp_column *a, const flsgpu_ffor_column *b,
                                       size_t n_pairs, double *d_results, uint32_t *d_medians,
                                       uint32_t *d_status, flsgpu_pair_query **out);
flsgpu_status flsgpu_pair_query_run(flsgpu_pair_query *q, flsgpu_stream stream);
flsgpu_status flsgpu_pair_query_capture_graph(flsgpu_pair_query *q, flsgpu_stream stream);
flsgpu_status flsgpu_pair_query_replay(flsgpu_pair_query *q, flsgpu_stream stream);
void flsgpu_pair_query_destroy(flsgpu_pair_query *q);

/* ---- GPU ALP encoder (f64) with the learned parameter proposal ---------
 * Replaces the reference's CPU alp::encode (src/alp/alp-bindings.cu:84-206)
 * for f64 columns.  Parameters are chosen per vector: mode 0 runs the plain
 * sampling search (all 190 (exponent, factor) pairs on the vector's 32
 * samples, estimate and tie rules of encoder.hpp:134-230); mode 1 asks the
 * network for its three best pairs, chooses among them with the reference's
 * second-level rule (encoder.hpp:237-300) and falls back to the plain search
 * when the choice leaves more than 30 exceptions (3%) in the vector (a
 * vector whose top proposal is ALP-RD is encoded with its best proposed ALP
 * pair under the same rule).  Exceptions store the original values, so the
 * column decodes exactly either way.  The network: 64 features of the 32
 * samples -> 128 -> 128 -> 192 logits (190 pairs, ALP-RD, padding), BF16
 * weights, FP32 accumulation on the tensor cores (tcgen05), trained on the
 * GPU with Adam on the plain search's labels. */
typedef struct flsgpu_alp_encoder flsgpu_alp_encoder;
typedef struct flsgpu_alp_encode_result {
  flsgpu_alp_column column;  /* device arrays in the encoder's workspace */
  size_t n_packed_words;
  size_t n_exceptions;
  size_t compressed_bytes;   /* reference accounting, alp-bindings.cu:19-43 */
  size_t n_fallback;         /* vectors that fell back to the plain search */
  size_t n_rd;               /* vectors whose search estimate calls for ALP-RD */
  double mean_bit_width;
} flsgpu_alp_encode_result;

flsgpu_status flsgpu_alp_encoder_create(uint32_t seed, flsgpu_alp_encoder **out);
void flsgpu_alp_encoder_destroy(flsgpu_alp_encoder *encoder);
/* Trains on the plain search's labels of d_values (n_values % 1024 == 0):
 * `epochs` passes of Adam over shuffled minibatches of `batch` rows
 * (batch % 128 == 0).  Synchronises; reports the first and last epoch's mean
 * cross entropy. */
flsgpu_status flsgpu_alp_encoder_train(flsgpu_alp_encoder *encoder, const double *d_values,
                                       size_t n_values, uint32_t epochs, uint32_t batch, float lr,
                                       float *h_loss_first, float *h_loss_last,
                                       flsgpu_stream stream);
flsgpu_status flsgpu_alp_encode_f64(flsgpu_alp_encoder *encoder, const double *d_values,
                                    size_t n_values, uint32_t mode,
                                    flsgpu_alp_encode_result *out, flsgpu_stream stream);
/* pieces exposed for tests and tools */
/* Top-k (k <= 4) proposed classes per vector in one fused kernel (features,
 * the three layers on the tensor cores with activations kept in shared
 * memory, top-k); _layered runs the same arithmetic as separate launches
 * (features, three GEMMs, top-k) and gives the same classes. */
flsgpu_status flsgpu_alp_encoder_propose(flsgpu_alp_encoder *encoder, const double *d_values,
                                         size_t n_values, uint32_t k, int16_t *d_cand,
                                         flsgpu_stream stream);
flsgpu_status flsgpu_alp_encoder_propose_layered(flsgpu_alp_encoder *encoder,
                                                 const double *d_values, size_t n_values,
                                                 uint32_t k, int16_t *d_cand,
                                                 flsgpu_stream stream);
flsgpu_status flsgpu_alp_plain_labels(const double *d_values, size_t n_values, int16_t *d_labels,
                                      int32_t *d_estimates, flsgpu_stream stream);
flsgpu_status flsgpu_alp_features(const double *d_values, size_t n_values, void *d_features_bf16,
                                  flsgpu_stream stream);
size_t flsgpu_alp_encoder_param_count(void);
flsgpu_status flsgpu_alp_encoder_get_params(const flsgpu_alp_encoder *encoder, float *h_params);
flsgpu_status flsgpu_alp_encoder_set_params(flsgpu_alp_encoder *encoder, const float *h_params);
flsgpu_status flsgpu_alp_encoder_gradients(flsgpu_alp_encoder *encoder, const void *d_features_bf16,
                                           const int16_t *d_labels, uint32_t rows, float *d_grads,
                                           float *h_loss, flsgpu_stream stream);
flsgpu_status flsgpu_alp_encoder_save(const flsgpu_alp_encoder *encoder, const char *path);
flsgpu_status flsgpu_alp_encoder_load(flsgpu_alp_encoder *encoder, const char *path);
/* The f32 GPU encoder: the float path of alp::encode (encoder.hpp:302-379,
 * alp-bindings.cu:84-206) with the pair chosen per vector by the plain
 * search (the 66 pairs 0 <= f <= e <= 10 on the vector's 32 samples, the
 * estimate and tie rules of find_top_k_combinations), exceptions and fill
 * of encode_simdized, FFOR at the signed minimum; an ALPColumn<float> in
 * the encoder's workspace (valid until its next encode).  n_rd counts the
 * vectors whose estimate reaches the ALP-RD limit (encoded as ALP all the
 * same).  Synchronises. */
flsgpu_status flsgpu_alp_encode_f32(flsgpu_alp_encoder *encoder, const float *d_values,
                                    size_t n_values, flsgpu_alp_encode_result *out,
                                    flsgpu_stream stream);

/* Hybrid encode: as flsgpu_alp_encode_f64, but the vectors that call for
 * ALP-RD are encoded as ALP-RD (upstream ALP switches scheme there,
 * src/alp/encoder.hpp:208-211, where the reference's alp::encode gives up)
 * into a flsgpu_alphybrid_column: mode 0 when the plain search's best
 * estimate reaches the ALP-RD limit (48 bits per value on the samples);
 * mode 1 when the network's top class is ALP-RD and none of its proposed ALP
 * pairs estimates below that limit on the samples, or when the plain search
 * of a fallback vector reaches it.  An ALP-RD vector carries a dictionary
 * of its own, built from its 32 samples with the cut search of
 * rd_encoder::init.  Decodes with flsgpu_decompress_alphybrid_f64. */
typedef struct flsgpu_alp_hybrid_encode_result {
  flsgpu_alphybrid_column column;  /* device arrays in the encoder's workspace */
  size_t n_alp_vectors, n_rd_vectors;
  size_t n_packed_words, n_exceptions;                  /* ALP part */
  size_t n_right_words, n_left_words, n_rd_exceptions;  /* ALP-RD part */
  size_t compressed_bytes;   /* ALP vectors as alp::encode accounts them, plus
                                the ALP-RD vectors (words, 4 B per exception,
                                48 B of dictionary and metadata) and one
                                scheme byte per vector */
  size_t n_fallback;         /* vectors that fell back to the plain search */
  double mean_bit_width;     /* over the ALP vectors */
  const uint8_t *d_flags;    /* per vector (device): bit 0 the plain search
                                ran as fallback, bit 1 encoded as ALP-RD */
} flsgpu_alp_hybrid_encode_result;
flsgpu_status flsgpu_alp_encode_hybrid_f64(flsgpu_alp_encoder *encoder, const double *d_values,
                                           size_t n_values, uint32_t mode,
                                           flsgpu_alp_hybrid_encode_result *out,
                                           flsgpu_stream stream);

/* ---- GPU ALP-RD encoder (rd_encoder::init / encode, src/alp/rd.hpp:
 *      28-140; the reference encodes ALP-RD on the CPU only and has no GPU
 *      ALP-RD format) ---------------------------------------------------------
 * One dictionary per rowgroup of rowgroup_vecs vectors (1..100; 100 is the
 * reference's ROWGROUP_SIZE, src/alp/config.hpp): the rowgroup's
 * first-level sample (every 12th vector, 32 values at stride 32 of each,
 * sampler.hpp:11-48) picks the cut (find_best_dictionary: right width 48..63
 * for f64, 16..31 for f32) and the <= 8 most frequent left parts (ties: the
 * smaller left part first); every vector is then split into right parts
 * (FastLanes lanes, FFOR base 0), dictionary indices (u16 FastLanes lanes at
 * width max(1, ceil(log2(dictionary size)))) and exceptions (left part +
 * position).  The column's arrays live in the encoder's workspace until its
 * next encode; it decodes with flsgpu_decompress_alprd_*.  n_values % 1024 ==
 * 0.  Synchronises (the sizes are read back). */
typedef struct flsgpu_alprd_encode_result {
  flsgpu_alprd_column column;
  size_t n_right_words;      /* right-part words, of the value's width */
  size_t n_left_words;       /* u16 words of dictionary indices */
  size_t n_exceptions;
  size_t n_dictionaries;     /* one per rowgroup */
  size_t compressed_bytes;   /* words + 4 B per exception + 16 B per dictionary
                                + 32 B of per-vector metadata */
} flsgpu_alprd_encode_result;
flsgpu_status flsgpu_alprd_encode_f64(flsgpu_alp_encoder *encoder, const double *d_values,
                                      size_t n_values, uint32_t rowgroup_vecs,
                                      flsgpu_alprd_encode_result *out, flsgpu_stream stream);
flsgpu_status flsgpu_alprd_encode_f32(flsgpu_alp_encoder *encoder, const float *d_values,
                                      size_t n_values, uint32_t rowgroup_vecs,
                                      flsgpu_alprd_encode_result *out, flsgpu_stream stream);

/* C (fp32 / bf16, M x N, row stride ldc) = A (bf16 M x K) . B (bf16 N x K)^T
 * [+ bias][relu] on the tensor cores (tcgen05, accumulator in TMEM);
 * N <= 256, K % 16 == 0, operands 16-byte aligned. */
flsgpu_status flsgpu_gemm_bf16_tn(const void *A, int lda, const void *B, int ldb, int M, int N,
                                  int K, float *Cf, void *Cb, int ldc, const float *bias, int relu,
                                  uint32_t *d_status, flsgpu_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* FLSGPU_B200_EXT_H */
