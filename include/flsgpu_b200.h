/*
 * flsgpu_b200.h -- C ABI of the B200 (sm_100a) FastLanes / ALP / ALP-RD
 * decoding library (libflsgpu_b200.so).
 *
 * Drop-in boundary for the decode path of SvenHepkema/msc-thesis-project:
 *   - column descriptors are field-for-field the reference's
 *     flsgpu::device column structs (src/flsgpu/structs.cuh:33-84);
 *   - every decode / query / compute entry point replaces one family of the
 *     reference's generated bindings (src/generated-bindings/
 *     kernel-bindings.cuh:11-175), which a C++ shim
 *     (msc-thesis-project_b200/cpp/flsgpu_bindings.hpp) re-exposes with the
 *     reference's own C++ signatures.
 *
 * Conventions
 *   - All pointers inside column descriptors and all d_* arguments are
 *     device pointers owned by the caller.  Host pointers are named h_*.
 *   - Output buffers must be 16-byte aligned (cudaMalloc memory is).
 *   - Entry points enqueue work on `stream` and return without
 *     synchronising, except where a comment says otherwise.
 *   - They return a flsgpu_status and never throw or exit (the reference
 *     exits the process on CUDA errors, src/flsgpu/host-utils.cuh:12-20,
 *     and throws std::invalid_argument on a missing binding,
 *     generate-kernel-bindings.py:209).  flsgpu_last_error() describes the
 *     last failure of the calling thread.
 *   - Reentrant; concurrent calls on different streams are independent.
 */
#ifndef FLSGPU_B200_H
#define FLSGPU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FLSGPU_B200_ABI_VERSION 1

typedef enum flsgpu_status {
  FLSGPU_OK = 0,
  FLSGPU_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad enum or size */
  FLSGPU_ERR_UNSUPPORTED = 2,      /* no kernel for this combination */
  FLSGPU_ERR_MISALIGNED = 3,       /* output or array not 16-byte aligned */
  FLSGPU_ERR_CORRUPT_COLUMN = 4,   /* device-side metadata check failed */
  FLSGPU_ERR_CUDA = 5,             /* CUDA runtime error */
  FLSGPU_ERR_TIMEOUT = 6,          /* a bounded device wait gave up */
  FLSGPU_ERR_OUT_OF_MEMORY = 7,
  FLSGPU_ERR_ENCODING = 8          /* data not ALP-encodable (alp::EncodingException) */
} flsgpu_status;

/* Same type as cudaStream_t; NULL is the legacy default stream. */
typedef struct CUstream_st *flsgpu_stream;

/* Device-side corruption flags OR-ed into flsgpu_decode_opts.d_status. */
#define FLSGPU_BAD_BIT_WIDTH 0x1u      /* bit width > bits of the type */
#define FLSGPU_BAD_OFFSET 0x2u         /* packed offset + size beyond bound */
#define FLSGPU_BAD_PARAMETER_INDEX 0x4u /* ALP factor / exponent index */
#define FLSGPU_BAD_EXCEPTION 0x8u      /* exception count / position range */
#define FLSGPU_WAIT_TIMEOUT 0x10u      /* a bounded device wait (staged copy) gave up */

/* reference enums::Unpacker (src/engine/enums.cuh:21-41), same order */
typedef enum flsgpu_unpacker {
  FLSGPU_UNPACKER_DUMMY = 0, FLSGPU_UNPACKER_OLD_FLS, FLSGPU_UNPACKER_SWITCH_CASE,
  FLSGPU_UNPACKER_STATELESS, FLSGPU_UNPACKER_STATELESS_BRANCHLESS,
  FLSGPU_UNPACKER_STATEFUL_CACHE, FLSGPU_UNPACKER_STATEFUL_LOCAL_1,
  FLSGPU_UNPACKER_STATEFUL_LOCAL_2, FLSGPU_UNPACKER_STATEFUL_LOCAL_4,
  FLSGPU_UNPACKER_STATEFUL_SHARED_1, FLSGPU_UNPACKER_STATEFUL_SHARED_2,
  FLSGPU_UNPACKER_STATEFUL_SHARED_4, FLSGPU_UNPACKER_STATEFUL_REGISTER_1,
  FLSGPU_UNPACKER_STATEFUL_REGISTER_2, FLSGPU_UNPACKER_STATEFUL_REGISTER_4,
  FLSGPU_UNPACKER_STATEFUL_REGISTER_BRANCHLESS_1,
  FLSGPU_UNPACKER_STATEFUL_REGISTER_BRANCHLESS_2,
  FLSGPU_UNPACKER_STATEFUL_REGISTER_BRANCHLESS_4,
  FLSGPU_UNPACKER_STATEFUL_BRANCHLESS,
  FLSGPU_UNPACKER_COUNT
} flsgpu_unpacker;

/* reference enums::Patcher (src/engine/enums.cuh:43-53), same order */
typedef enum flsgpu_patcher {
  FLSGPU_PATCHER_NONE = 0, FLSGPU_PATCHER_DUMMY, FLSGPU_PATCHER_STATELESS,
  FLSGPU_PATCHER_STATEFUL, FLSGPU_PATCHER_NAIVE, FLSGPU_PATCHER_NAIVE_BRANCHLESS,
  FLSGPU_PATCHER_PREFETCH_POSITION, FLSGPU_PATCHER_PREFETCH_ALL,
  FLSGPU_PATCHER_PREFETCH_ALL_BRANCHLESS,
  FLSGPU_PATCHER_COUNT
} flsgpu_patcher;

/* B200 kernel variants of the full decompression (no reference
 * counterpart: the reference picks an unpacker per launch, this library a
 * register budget).  Both decode every width with the same unpackers. */
typedef enum flsgpu_variant {
  FLSGPU_VARIANT_AUTO = 0,       /* the tuned choice for the column's value
                                    type and kind (flsgpu_tuning_*) */
  FLSGPU_VARIANT_REGS = 1,       /* register-rich: 2 resident blocks per SM
                                    for 32-bit lanes, 1 for 64-bit lanes */
  FLSGPU_VARIANT_OCCUPANCY = 2,  /* register-capped for twice the resident
                                    blocks (more loads in flight) */
  FLSGPU_VARIANT_STAGED = 3,     /* 64-bit lanes: each vector's packed words
                                    (width <= 32) copied into a per-warp
                                    shared-memory slot by a bulk copy one
                                    vector ahead, unpacked from there; other
                                    widths and 32-bit lanes as REGS */
  FLSGPU_VARIANT_COUNT
} flsgpu_variant;

/* ---- column descriptors (reference src/flsgpu/structs.cuh:33-84) ----- */
typedef struct flsgpu_bp_column {      /* device::BPColumn<T> :33 */
  size_t n_values;
  size_t n_vecs;
  void *packed_array;                  /* UINT_T lanes, FastLanes layout */
  uint8_t *bit_widths;                 /* per vector */
  size_t *vector_offsets;              /* per vector, in UINT_T words */
} flsgpu_bp_column;

typedef struct flsgpu_ffor_column {    /* device::FFORColumn<T> :43 */
  size_t n_values;
  flsgpu_bp_column bp;
  void *bases;                         /* UINT_T per vector */
} flsgpu_ffor_column;

typedef struct flsgpu_alp_column {     /* device::ALPColumn<T> :50 */
  size_t n_values;
  flsgpu_ffor_column ffor;             /* encoded integers as UINT_T */
  void *factors;                       /* INT_T[19 | 10], NULL = built-in */
  void *fractions;                     /* T[21 | 11],     NULL = built-in */
  uint8_t *factor_indices;
  uint8_t *fraction_indices;
  size_t n_exceptions;
  size_t *exceptions_offsets;          /* per vector */
  void *exceptions;                    /* T, original values */
  uint16_t *positions;                 /* ascending within a vector */
  uint16_t *counts;                    /* per vector */
} flsgpu_alp_column;

typedef struct flsgpu_alpx_column {    /* device::ALPExtendedColumn<T> :68 */
  size_t n_values;
  flsgpu_ffor_column ffor;
  void *factors;
  void *fractions;
  uint8_t *factor_indices;
  uint8_t *fraction_indices;
  size_t n_exceptions;
  size_t *exceptions_offsets;          /* per vector */
  void *exceptions;                    /* grouped by lane within a vector */
  uint16_t *positions;
  uint16_t *offsets_counts;            /* per vector x lane: count<<10 | offset */
} flsgpu_alpx_column;

/* ALP-RD (no GPU format in the reference; decode restates
 * src/alp/rd.hpp:146-172).  Right parts are FastLanes-packed UINT_T words
 * (FFOR base 0) at right_bw = right.bit_widths[vi]; left parts are
 * dictionary indices packed as u16 FastLanes lanes at left.bit_widths[vi]
 * (<= 3); dictionary d is dictionaries[8*d .. 8*d+7]; vector vi uses
 * dictionary dictionary_indices[vi].  Exceptions hold the full left part of
 * values whose left part is not in the dictionary. */
typedef struct flsgpu_alprd_column {
  size_t n_values;
  flsgpu_bp_column right;
  flsgpu_bp_column left;
  uint16_t *dictionaries;
  uint32_t *dictionary_indices;
  size_t n_exceptions;
  size_t *exceptions_offsets;
  uint16_t *exceptions;
  uint16_t *positions;
  uint16_t *counts;
} flsgpu_alprd_column;

/* Hybrid ALP / ALP-RD column (no counterpart in the reference, whose
 * alp::encode rejects data that calls for ALP-RD; upstream ALP picks the
 * scheme per rowgroup, src/alp/encoder.hpp:208-211): vector v is decoded
 * from `alp` when schemes[v] == FLSGPU_SCHEME_ALP and from `rd` when
 * schemes[v] == FLSGPU_SCHEME_ALP_RD.  Both sub-columns index every vector;
 * a vector's entry in the other sub-column is empty (width 0, no
 * exceptions, no packed words). */
#define FLSGPU_SCHEME_ALP 0u
#define FLSGPU_SCHEME_ALP_RD 1u
typedef struct flsgpu_alphybrid_column {
  size_t n_values;
  flsgpu_alp_column alp;
  flsgpu_alprd_column rd;
  uint8_t *schemes;                    /* per vector */
} flsgpu_alphybrid_column;

typedef struct flsgpu_decode_opts {
  uint32_t unpack_n_vectors;  /* reference UNPACK_N_VECTORS (1, 4): advisory */
  uint32_t unpack_n_values;   /* reference UNPACK_N_VALUES (1, 32): advisory */
  uint32_t unpacker;          /* flsgpu_unpacker; every value decodes
                                 correctly, DUMMY included */
  uint32_t patcher;           /* flsgpu_patcher; NONE/DUMMY skip patching */
  uint32_t variant;           /* flsgpu_variant */
  uint32_t reserved;
  uint32_t *d_status;         /* optional: device word OR-ed with FLSGPU_BAD_* */
  size_t n_packed_values;     /* optional bound of packed_array (0: none) */
} flsgpu_decode_opts;

/* ---- library --------------------------------------------------------- */
uint32_t flsgpu_abi_version(void);
const char *flsgpu_last_error(void);
/* Number of __global__ kernels this library launched since load (all
 * threads), for launch accounting in benchmarks. */
uint64_t flsgpu_launch_count(void);

/* ---- full decompression (kernels::device::decompress_column,
 *      src/engine/kernels.cuh:13-32; bindings::decompress_column,
 *      kernel-bindings.cuh:42-90).  d_out receives n_values elements in
 *      row order; the reference's tail-vector drop is not reproduced. ---- */
flsgpu_status flsgpu_decompress_bp_u32(const flsgpu_bp_column *column, uint32_t *d_out,
                                       const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_bp_u64(const flsgpu_bp_column *column, uint64_t *d_out,
                                       const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_ffor_u32(const flsgpu_ffor_column *column, uint32_t *d_out,
                                         const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_ffor_u64(const flsgpu_ffor_column *column, uint64_t *d_out,
                                         const flsgpu_decode_opts *opts, flsgpu_stream stream);
/* 8- and 16-bit lanes (fls::unpack / fls::unffor for uint8_t / uint16_t,
 * src/fls/fls-bindings.hpp:8-52, CPU-only in the reference): the same
 * descriptors with packed_array holding u8 / u16 lane words (128 / 64 lanes
 * per vector), vector_offsets in those words, bases u8 / u16; packed words
 * and output 4-byte aligned. */
flsgpu_status flsgpu_decompress_bp_u8(const flsgpu_bp_column *column, uint8_t *d_out,
                                      const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_bp_u16(const flsgpu_bp_column *column, uint16_t *d_out,
                                       const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_ffor_u8(const flsgpu_ffor_column *column, uint8_t *d_out,
                                        const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_ffor_u16(const flsgpu_ffor_column *column, uint16_t *d_out,
                                         const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_alp_f32(const flsgpu_alp_column *column, float *d_out,
                                        const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_alp_f64(const flsgpu_alp_column *column, double *d_out,
                                        const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_alpx_f32(const flsgpu_alpx_column *column, float *d_out,
                                         const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_alpx_f64(const flsgpu_alpx_column *column, double *d_out,
                                         const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_alprd_f32(const flsgpu_alprd_column *column, float *d_out,
                                          const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_decompress_alprd_f64(const flsgpu_alprd_column *column, double *d_out,
                                          const flsgpu_decode_opts *opts, flsgpu_stream stream);

flsgpu_status flsgpu_decompress_alphybrid_f32(const flsgpu_alphybrid_column *column,
                                              float *d_out, const flsgpu_decode_opts *opts,
                                              flsgpu_stream stream);
flsgpu_status flsgpu_decompress_alphybrid_f64(const flsgpu_alphybrid_column *column,
                                              double *d_out, const flsgpu_decode_opts *opts,
                                              flsgpu_stream stream);

/* ---- lane-divided exception layout on the GPU
 *      (host::ALPColumn::create_extended_column and
 *      convert_exceptions_to_lane_divided_format, src/flsgpu/structs.cuh:
 *      231-308, which the reference runs on the host).  Writes the
 *      exceptions of `src` regrouped by FastLanes lane (order kept within a
 *      lane) to d_exceptions / d_positions (src->n_exceptions elements each)
 *      and per vector and lane (count << 10) | offset to d_offsets_counts
 *      (n_vecs * 32 (f32) or * 16 (f64) elements; 16 bits, so a 64-bit lane
 *      with 64 exceptions wraps as in the reference), and fills *dst: the
 *      extended column sharing src's packed words, metadata and exception
 *      offsets.  Enqueued on `stream`. ------------------------------------ */
flsgpu_status flsgpu_alp_to_extended_f32(const flsgpu_alp_column *src, float *d_exceptions,
                                         uint16_t *d_positions, uint16_t *d_offsets_counts,
                                         flsgpu_alpx_column *dst, flsgpu_stream stream);
flsgpu_status flsgpu_alp_to_extended_f64(const flsgpu_alp_column *src, double *d_exceptions,
                                         uint16_t *d_positions, uint16_t *d_offsets_counts,
                                         flsgpu_alpx_column *dst, flsgpu_stream stream);

/* ---- FastLanes packing, the encoder side (fls::ffor src/fls/ffor.cpp:
 *      29861, fls::pack src/fls/pack.cpp:29731, base / width rule of
 *      analyze_ffor src/alp/encoder.hpp:104-115; the reference packs on the
 *      CPU, vector by vector).  n_values % 1024 == 0.  Per vector: the base
 *      (base_mode FLSGPU_BASE_MIN: unsigned minimum; FLSGPU_BASE_SIGNED_MIN:
 *      minimum as a signed integer, as analyze_ffor; FLSGPU_BASE_ZERO: 0,
 *      i.e. BP, d_bases may be NULL), the width bits(max - base), and the
 *      packed words at d_vector_offsets[v] (exclusive prefix of width x
 *      lanes).  d_packed must hold n_values elements (the widest case);
 *      d_n_packed (optional, device) receives the number of packed words.
 *      Output decodes with flsgpu_decompress_{ffor,bp}_* and is word for
 *      word what fls::ffor / fls::pack write. ---- */
#define FLSGPU_BASE_MIN 0u
#define FLSGPU_BASE_SIGNED_MIN 1u
#define FLSGPU_BASE_ZERO 2u
flsgpu_status flsgpu_ffor_encode_u8(const uint8_t *d_values, size_t n_values, uint32_t base_mode,
                                    uint8_t *d_packed, uint8_t *d_bit_widths,
                                    uint64_t *d_vector_offsets, uint8_t *d_bases,
                                    uint64_t *d_n_packed, flsgpu_stream stream);
flsgpu_status flsgpu_ffor_encode_u16(const uint16_t *d_values, size_t n_values, uint32_t base_mode,
                                     uint16_t *d_packed, uint8_t *d_bit_widths,
                                     uint64_t *d_vector_offsets, uint16_t *d_bases,
                                     uint64_t *d_n_packed, flsgpu_stream stream);
flsgpu_status flsgpu_ffor_encode_u32(const uint32_t *d_values, size_t n_values, uint32_t base_mode,
                                     uint32_t *d_packed, uint8_t *d_bit_widths,
                                     uint64_t *d_vector_offsets, uint32_t *d_bases,
                                     uint64_t *d_n_packed, flsgpu_stream stream);
flsgpu_status flsgpu_ffor_encode_u64(const uint64_t *d_values, size_t n_values, uint32_t base_mode,
                                     uint64_t *d_packed, uint8_t *d_bit_widths,
                                     uint64_t *d_vector_offsets, uint64_t *d_bases,
                                     uint64_t *d_n_packed, flsgpu_stream stream);

/* ---- decode fused with a sum (model: kernels::device::query_column,
 *      kernels.cuh:34-54).  Integer sums are exact mod 2^64.  Float sums
 *      use a fixed reduction tree (per-lane ascending, warp butterfly,
 *      pairwise over vectors) so results are reproducible bit for bit;
 *      d_partials is caller workspace of flsgpu_sum_workspace_f64(n_values)
 *      doubles; on return d_partials[0 .. n_vecs) hold the per-vector sums
 *      only when n_vecs <= 2048. */
size_t flsgpu_sum_workspace_f64(size_t n_values);
flsgpu_status flsgpu_sum_ffor_u32(const flsgpu_ffor_column *column, uint64_t *d_sum,
                                  const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_sum_ffor_u64(const flsgpu_ffor_column *column, uint64_t *d_sum,
                                  const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_sum_alp_f64(const flsgpu_alp_column *column, double *d_sum,
                                 double *d_partials, const flsgpu_decode_opts *opts,
                                 flsgpu_stream stream);
flsgpu_status flsgpu_sum_alpx_f64(const flsgpu_alpx_column *column, double *d_sum,
                                  double *d_partials, const flsgpu_decode_opts *opts,
                                  flsgpu_stream stream);

/* Decode-and-sum of an f64 ALP column that allocates nothing.  No
 * counterpart in the reference.  For callers that cannot provide device
 * memory (an engine with its own fixed memory budget, a thread capturing a
 * CUDA graph, a plug-in that must not touch the host process's allocator):
 * the scratch of the fixed reduction tree lives in a static device array of
 * FLSGPU_NOALLOC_MAX_VECTORS vectors (2 MiB), reserved on every GPU that
 * loads the library until the process exits.  Same result, bit for bit, as
 * flsgpu_sum_alp_f64.  Columns of more vectors are rejected with
 * FLSGPU_ERR_INVALID_ARGUMENT.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture.  All calls on a device share the array: calls whose
 * kernels overlap on the GPU race, so serialise them. */
#define FLSGPU_NOALLOC_MAX_VECTORS 262144
flsgpu_status flsgpu_sum_alp_f64_noalloc(const flsgpu_alp_column *column, double *d_sum,
                                         const flsgpu_decode_opts *opts, flsgpu_stream stream);

/* ---- magic-value scan (kernels::device::query_column, kernels.cuh:34-54;
 *      bindings::query_column, kernel-bindings.cuh:92-131).  *d_found is
 *      set to 1 when some decoded value equals `magic` (float compare) and
 *      is left untouched otherwise: clear it first. ---------------------- */
flsgpu_status flsgpu_query_bp_u32(const flsgpu_bp_column *column, uint32_t magic, uint8_t *d_found,
                                  const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_query_bp_u64(const flsgpu_bp_column *column, uint64_t magic, uint8_t *d_found,
                                  const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_query_ffor_u32(const flsgpu_ffor_column *column, uint32_t magic,
                                    uint8_t *d_found, const flsgpu_decode_opts *opts,
                                    flsgpu_stream stream);
flsgpu_status flsgpu_query_ffor_u64(const flsgpu_ffor_column *column, uint64_t magic,
                                    uint8_t *d_found, const flsgpu_decode_opts *opts,
                                    flsgpu_stream stream);
flsgpu_status flsgpu_query_alp_f32(const flsgpu_alp_column *column, float magic, uint8_t *d_found,
                                   const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_query_alp_f64(const flsgpu_alp_column *column, double magic, uint8_t *d_found,
                                   const flsgpu_decode_opts *opts, flsgpu_stream stream);
flsgpu_status flsgpu_query_alpx_f32(const flsgpu_alpx_column *column, float magic,
                                    uint8_t *d_found, const flsgpu_decode_opts *opts,
                                    flsgpu_stream stream);
flsgpu_status flsgpu_query_alpx_f64(const flsgpu_alpx_column *column, double magic,
                                    uint8_t *d_found, const flsgpu_decode_opts *opts,
                                    flsgpu_stream stream);

/* ---- synthetic ALU load (kernels::device::compute_column,
 *      kernels.cuh:56-89; bindings::compute_column, kernel-bindings.cuh:
 *      133-144).  Writes 1 to *d_out when a lane ends all-ones (never, as in
 *      the reference, since the last step ANDs with zero). ---------------- */
flsgpu_status flsgpu_compute_ffor_u32(const flsgpu_ffor_column *column, uint32_t n_repetitions,
                                      uint8_t *d_out, const flsgpu_decode_opts *opts,
                                      flsgpu_stream stream);
flsgpu_status flsgpu_compute_ffor_u64(const flsgpu_ffor_column *column, uint32_t n_repetitions,
                                      uint8_t *d_out, const flsgpu_decode_opts *opts,
                                      flsgpu_stream stream);

/* ---- multi-column conjunctive scan (multi_column::query_multi_column,
 *      src/generated-bindings/multi-column-device-kernels.cuh:11-439).
 *      *d_out is set to 1 when, for some vector lane, every value of that
 *      lane in every column equals `value`.  1 <= n_columns <= 16. ------- */
flsgpu_status flsgpu_query_multi_column_ffor_u32(const flsgpu_ffor_column *columns,
                                                 uint32_t n_columns, uint32_t value,
                                                 uint8_t *d_out, const flsgpu_decode_opts *opts,
                                                 flsgpu_stream stream);
flsgpu_status flsgpu_query_multi_column_ffor_u64(const flsgpu_ffor_column *columns,
                                                 uint32_t n_columns, uint64_t value,
                                                 uint8_t *d_out, const flsgpu_decode_opts *opts,
                                                 flsgpu_stream stream);
flsgpu_status flsgpu_query_multi_column_alp_f32(const flsgpu_alp_column *columns,
                                                uint32_t n_columns, float value, uint8_t *d_out,
                                                const flsgpu_decode_opts *opts,
                                                flsgpu_stream stream);
flsgpu_status flsgpu_query_multi_column_alp_f64(const flsgpu_alp_column *columns,
                                                uint32_t n_columns, double value,
                                                uint8_t *d_out, const flsgpu_decode_opts *opts,
                                                flsgpu_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* FLSGPU_B200_H */
