/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's FastLanes / ALP / ALP-RD algorithms
 * (SvenHepkema/msc-thesis-project, files cited per function in oracle.c).
 * It is the checker for tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs, and nothing else: the product
 * library (msc-thesis-project_b200/) never links, loads or calls it.
 *
 * Parity pinning: tests/test_oracle.py checks every function here against
 * golden vectors produced by the reference's own CPU code (oracle/_ref,
 * compiled from the reference sources by oracle/build_ref.sh), committed
 * under tests/golden/.
 */
#ifndef FLS_ORACLE_H
#define FLS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- FastLanes 1024-value vectors (one vector per call) ---------------- */
void orc_pack_u16(const uint16_t *in, uint16_t *out, int bw);
void orc_pack_u32(const uint32_t *in, uint32_t *out, int bw);
void orc_pack_u64(const uint64_t *in, uint64_t *out, int bw);
void orc_unpack_u16(const uint16_t *in, uint16_t *out, int bw);
void orc_unpack_u32(const uint32_t *in, uint32_t *out, int bw);
void orc_unpack_u64(const uint64_t *in, uint64_t *out, int bw);
void orc_pack_u8(const uint8_t *in, uint8_t *out, int bw);
void orc_unpack_u8(const uint8_t *in, uint8_t *out, int bw);
void orc_ffor_u8(const uint8_t *in, uint8_t *out, int bw, uint8_t base);
void orc_ffor_u16(const uint16_t *in, uint16_t *out, int bw, uint16_t base);
void orc_unffor_u8(const uint8_t *in, uint8_t *out, int bw, uint8_t base);
void orc_unffor_u16(const uint16_t *in, uint16_t *out, int bw, uint16_t base);
void orc_ffor_u32(const uint32_t *in, uint32_t *out, int bw, uint32_t base);
void orc_ffor_u64(const uint64_t *in, uint64_t *out, int bw, uint64_t base);
void orc_unffor_u32(const uint32_t *in, uint32_t *out, int bw, uint32_t base);
void orc_unffor_u64(const uint64_t *in, uint64_t *out, int bw, uint64_t base);

/* ---- ALP vector decode: unFFOR + scale (falp) -------------------------- */
void orc_falp_f32(const uint32_t *in, float *out, int bw, uint32_t base,
                  int fac, int exp);
void orc_falp_f64(const uint64_t *in, double *out, int bw, uint64_t base,
                  int fac, int exp);

/* ---- column-level decode (vector loop, as the reference's data.cuh) ---- */
void orc_decode_bp_u32(const uint32_t *packed, const uint8_t *bw,
                       const size_t *offs, size_t n_vecs, uint32_t *out);
void orc_decode_bp_u64(const uint64_t *packed, const uint8_t *bw,
                       const size_t *offs, size_t n_vecs, uint64_t *out);
void orc_decode_ffor_u32(const uint32_t *packed, const uint8_t *bw,
                         const size_t *offs, const uint32_t *bases,
                         size_t n_vecs, uint32_t *out);
void orc_decode_ffor_u64(const uint64_t *packed, const uint8_t *bw,
                         const size_t *offs, const uint64_t *bases,
                         size_t n_vecs, uint64_t *out);
/* ALPColumn: counts[vi]; ALPExtendedColumn: counts == NULL and
 * offsets_counts != NULL (count of a vector = sum over lanes of oc >> 10). */
void orc_decode_alp_f32(const uint32_t *packed, const uint8_t *bw,
                        const size_t *offs, const uint32_t *bases,
                        const uint8_t *fac, const uint8_t *exp,
                        const size_t *exc_offs, const float *exc,
                        const uint16_t *pos, const uint16_t *counts,
                        const uint16_t *offsets_counts, size_t n_vecs,
                        float *out);
void orc_decode_alp_f64(const uint64_t *packed, const uint8_t *bw,
                        const size_t *offs, const uint64_t *bases,
                        const uint8_t *fac, const uint8_t *exp,
                        const size_t *exc_offs, const double *exc,
                        const uint16_t *pos, const uint16_t *counts,
                        const uint16_t *offsets_counts, size_t n_vecs,
                        double *out);

/* Lane-divided ("extended") exception layout, structs.cuh:231-306.
 * Returns the number of lanes whose 6-bit count field overflowed. */
size_t orc_alp_to_extended(int type_bits, const void *exc, const uint16_t *pos,
                           const uint16_t *counts, size_t n_vecs,
                           void *out_exc, uint16_t *out_pos,
                           uint16_t *out_offsets_counts);

/* ---- ALP encoder (plain sampling search) ------------------------------- */
/* Output buffers are sized by the caller for the worst case:
 *   packed: n_vecs*1024 words, exceptions/positions: n_vecs*1024.
 * rowgroup_vecs == 0: one sampling state for the whole column (the
 * reference's alp::encode); otherwise one state per rowgroup_vecs vectors.
 * Returns 0 on success, 1 when sampling selects ALP-RD (the reference's
 * EncodingException), with *rd_rowgroup set to the failing rowgroup. */
typedef struct {
  size_t n_packed;      /* words written to packed */
  size_t n_exceptions;  /* total exceptions */
  size_t compressed_bytes;          /* reference accounting, ALPColumn */
  size_t compressed_bytes_extended; /* reference accounting, extended */
  size_t rd_rowgroup;
} orc_alp_encode_info;

int orc_alp_encode_f64(const double *in, size_t n_vecs, size_t rowgroup_vecs,
                       uint64_t *packed, uint8_t *bw, size_t *offs,
                       uint64_t *bases, uint8_t *fac, uint8_t *exp,
                       size_t *exc_offs, double *exc, uint16_t *pos,
                       uint16_t *counts, orc_alp_encode_info *info);
int orc_alp_encode_f32(const float *in, size_t n_vecs, size_t rowgroup_vecs,
                       uint32_t *packed, uint8_t *bw, size_t *offs,
                       uint32_t *bases, uint8_t *fac, uint8_t *exp,
                       size_t *exc_offs, float *exc, uint16_t *pos,
                       uint16_t *counts, orc_alp_encode_info *info);

/* Sampling search pieces, exposed for label generation and unit tests.
 * top-k over a rowgroup sample: writes up to 5 (exp, fac) pairs, returns k,
 * or -1 when the rowgroup should use ALP-RD. */
int orc_alp_rowgroup_topk_f64(const double *rowgroup, size_t n_values,
                              uint8_t *k_exp, uint8_t *k_fac);
int orc_alp_rowgroup_topk_f32(const float *rowgroup, size_t n_values,
                              uint8_t *k_exp, uint8_t *k_fac);
/* 1: rowgroups at the ALP-RD limit keep their ALP top-k (ALP-only encoder);
 * 0 (default): they are rejected as alp::encode rejects them. */
void orc_set_rd_as_alp(int on);
/* Per-vector exhaustive search: top-k restricted to one vector's 32
 * samples (every 32nd value).  Returns the packed label e*32+f, or -1 when
 * no pair has >= 2 non-exceptions or the estimate crosses the RD limit.
 * est_bits receives the estimated sample bits of the chosen pair. */
int orc_alp_vector_best_f64(const double *vec, uint64_t *est_bits);
/* f32: the best pair of the vector's 32 samples (returned even where the
 * estimate reaches the ALP-RD limit), e*32+f; and one vector's encode. */
int orc_alp_vector_best_f32(const float *vec, uint64_t *est_bits);
int orc_alp_encode_vector_f32(const float *vec, int exp, int fac, int32_t *encoded, float *exc,
                              uint16_t *pos);
/* second-level choice for one vector among k candidates */
void orc_alp_vector_choose_f64(const double *vec, int k, const uint8_t *k_exp,
                               const uint8_t *k_fac, uint8_t *exp,
                               uint8_t *fac);
/* Encode one vector with a given (exp, fac); returns exception count. */
int orc_alp_encode_vector_f64(const double *vec, int exp, int fac,
                              int64_t *encoded, double *exc, uint16_t *pos);

/* ---- ALP-RD ------------------------------------------------------------ */
typedef struct {
  uint8_t right_bw;
  uint8_t left_bw;
  uint8_t dict_size;
  uint16_t dict[8];
} orc_rd_state;
void orc_rd_init_f64(const double *rowgroup, size_t n_values, orc_rd_state *st);
void orc_rd_init_f32(const float *rowgroup, size_t n_values, orc_rd_state *st);
/* encode one vector: right parts (1024), left dictionary indices (1024),
 * exceptions (left part + position); returns exception count */
int orc_rd_encode_vector_f64(const double *vec, const orc_rd_state *st,
                             uint64_t *right, uint16_t *left_idx,
                             uint16_t *exc, uint16_t *pos);
int orc_rd_encode_vector_f32(const float *vec, const orc_rd_state *st,
                             uint32_t *right, uint16_t *left_idx,
                             uint16_t *exc, uint16_t *pos);
void orc_rd_decode_vector_f64(const uint64_t *right, const uint16_t *left_idx,
                              const uint16_t *dict, int right_bw,
                              const uint16_t *exc, const uint16_t *pos,
                              int n_exc, double *out);
void orc_rd_decode_vector_f32(const uint32_t *right, const uint16_t *left_idx,
                              const uint16_t *dict, int right_bw,
                              const uint16_t *exc, const uint16_t *pos,
                              int n_exc, float *out);
/* column-level RD decode of the library's packed RD column format */
void orc_decode_rd_f64(const uint64_t *right_packed, const size_t *right_offs,
                       const uint8_t *right_bw, const uint16_t *left_packed,
                       const size_t *left_offs, const uint8_t *left_bw,
                       const uint16_t *dicts, const uint32_t *dict_index,
                       const size_t *exc_offs, const uint16_t *exc,
                       const uint16_t *pos, const uint16_t *counts,
                       size_t n_vecs, double *out);
void orc_decode_rd_f32(const uint32_t *right_packed, const size_t *right_offs,
                       const uint8_t *right_bw, const uint16_t *left_packed,
                       const size_t *left_offs, const uint8_t *left_bw,
                       const uint16_t *dicts, const uint32_t *dict_index,
                       const size_t *exc_offs, const uint16_t *exc,
                       const uint16_t *pos, const uint16_t *counts,
                       size_t n_vecs, float *out);

/* ---- fixed-tree reductions (the order the GPU kernels use) ------------- */
/* Per vector: lane l sums its values k = 0..VPL-1 in order; lanes are then
 * combined by the butterfly l ^ 16, l ^ 8, ... (f64) -> one partial per
 * vector; partials are combined pairwise (stride doubling) over vectors. */
double orc_tree_sum_f64(const double *values, size_t n_vecs);
double orc_tree_sum_masked_f64(const double *values, const uint32_t *keys,
                               uint32_t threshold, size_t n_vecs);
float orc_tree_sum_f32(const float *values, size_t n_vecs);
uint64_t orc_sum_u32(const uint32_t *values, size_t n);
uint64_t orc_sum_u64(const uint64_t *values, size_t n);
/* lower median: element of rank floor((n-1)/2) */
uint32_t orc_median_u32(const uint32_t *values, size_t n);

#ifdef __cplusplus
}
#endif
#endif
