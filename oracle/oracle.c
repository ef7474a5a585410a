/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Plain-C restatement of the reference's CPU codecs.  Every routine cites
 * the reference file:line whose behaviour it restates.  Compile with
 * -O2 -ffp-contract=off and without -ffast-math / -march=native: the ALP
 * encoder's "x * 10^e * 10^-f + MAGIC - MAGIC" must not be contracted into
 * an FMA (reference src/alp/encoder.hpp:78-83).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define VEC 1024

/* ---------------------------------------------------------------------- */
/* FastLanes interleaved layout.                                           */
/* A vector of 1024 values of a TB-bit type is N = 1024/TB lanes of TB     */
/* values; value k of lane l is element l + k*N (reference                 */
/* src/fls/unffor.cpp:2243-2362, out index (i*1) + (32*k)).  Each lane's   */
/* values form one LSB-first bit stream of k*bw bits whose TB-bit word j   */
/* is stored at packed[j*N + l] (unffor.cpp:2252, in + (0*32) + i + 32*j). */
/* ---------------------------------------------------------------------- */

static inline uint64_t mask_bits(int bw) {
  return bw >= 64 ? ~(uint64_t)0 : (((uint64_t)1 << bw) - 1);
}

#define DEFINE_FLS(TB, UT)                                                   \
  static inline uint64_t read_word_##TB(const UT *in, int j, int l) {        \
    return (uint64_t)in[j * (VEC / TB) + l];                                 \
  }                                                                          \
  void orc_unpack_u##TB(const UT *in, UT *out, int bw) {                     \
    const int N = VEC / TB;                                                  \
    const uint64_t m = mask_bits(bw);                                        \
    for (int l = 0; l < N; ++l) {                                            \
      for (int k = 0; k < TB; ++k) {                                         \
        uint64_t v = 0;                                                      \
        if (bw > 0) {                                                        \
          const int start = k * bw;                                          \
          const int j = start / TB, off = start % TB;                        \
          v = read_word_##TB(in, j, l) >> off;                               \
          if (off + bw > TB) v |= read_word_##TB(in, j + 1, l) << (TB - off); \
          v &= m;                                                            \
        }                                                                    \
        out[l + k * N] = (UT)v;                                              \
      }                                                                      \
    }                                                                        \
  }                                                                          \
  void orc_pack_u##TB(const UT *in, UT *out, int bw) {                       \
    const int N = VEC / TB;                                                  \
    const uint64_t m = mask_bits(bw);                                        \
    if (bw == 0) return;                                                     \
    memset(out, 0, sizeof(UT) * (size_t)N * (size_t)bw);                     \
    for (int l = 0; l < N; ++l) {                                            \
      for (int k = 0; k < TB; ++k) {                                         \
        const uint64_t v = (uint64_t)in[l + k * N] & m;                      \
        const int start = k * bw;                                            \
        const int j = start / TB, off = start % TB;                          \
        out[j * N + l] |= (UT)(v << off);                                    \
        if (off + bw > TB) out[(j + 1) * N + l] |= (UT)(v >> (TB - off));    \
      }                                                                      \
    }                                                                        \
  }

DEFINE_FLS(8, uint8_t)
DEFINE_FLS(16, uint16_t)
DEFINE_FLS(32, uint32_t)
DEFINE_FLS(64, uint64_t)

/* fls::ffor packs (in - base) (src/fls/ffor.cpp:29861); fls::unffor adds
 * the base back with unsigned wraparound (src/fls/unffor.cpp:22901). */
void orc_ffor_u8(const uint8_t *in, uint8_t *out, int bw, uint8_t base) {
  uint8_t tmp[VEC];
  for (int i = 0; i < VEC; ++i) tmp[i] = (uint8_t)(in[i] - base);
  orc_pack_u8(tmp, out, bw);
}
void orc_ffor_u16(const uint16_t *in, uint16_t *out, int bw, uint16_t base) {
  uint16_t tmp[VEC];
  for (int i = 0; i < VEC; ++i) tmp[i] = (uint16_t)(in[i] - base);
  orc_pack_u16(tmp, out, bw);
}
void orc_unffor_u8(const uint8_t *in, uint8_t *out, int bw, uint8_t base) {
  orc_unpack_u8(in, out, bw);
  for (int i = 0; i < VEC; ++i) out[i] = (uint8_t)(out[i] + base);
}
void orc_unffor_u16(const uint16_t *in, uint16_t *out, int bw, uint16_t base) {
  orc_unpack_u16(in, out, bw);
  for (int i = 0; i < VEC; ++i) out[i] = (uint16_t)(out[i] + base);
}
void orc_ffor_u32(const uint32_t *in, uint32_t *out, int bw, uint32_t base) {
  uint32_t tmp[VEC];
  for (int i = 0; i < VEC; ++i) tmp[i] = in[i] - base;
  orc_pack_u32(tmp, out, bw);
}
void orc_ffor_u64(const uint64_t *in, uint64_t *out, int bw, uint64_t base) {
  uint64_t tmp[VEC];
  for (int i = 0; i < VEC; ++i) tmp[i] = in[i] - base;
  orc_pack_u64(tmp, out, bw);
}
void orc_unffor_u32(const uint32_t *in, uint32_t *out, int bw, uint32_t base) {
  orc_unpack_u32(in, out, bw);
  for (int i = 0; i < VEC; ++i) out[i] += base;
}
void orc_unffor_u64(const uint64_t *in, uint64_t *out, int bw, uint64_t base) {
  orc_unpack_u64(in, out, bw);
  for (int i = 0; i < VEC; ++i) out[i] += base;
}

/* ---------------------------------------------------------------------- */
/* ALP constants, src/alp/constants.hpp:49-55 (float), :76-144 (double).   */
/* ---------------------------------------------------------------------- */
static const float F32_FRAC[11] = {1.0f,  0.1f,  0.01f, 0.001f, 0.0001f,
                                   1e-5f, 1e-6f, 1e-7f, 1e-8f,  1e-9f,
                                   1e-10f};
static const float F32_EXP[11] = {1.0f, 10.0f, 100.0f, 1000.0f, 10000.0f,
                                  1e5f, 1e6f,  1e7f,   1e8f,    1e9f,
                                  1e10f};
static const int32_t F32_FACT[10] = {1,      10,      100,      1000,
                                     10000,  100000,  1000000,  10000000,
                                     100000000, 1000000000};
static const double F64_FRAC[21] = {
    1.0,   0.1,   0.01,  0.001, 0.0001, 1e-5,  1e-6,  1e-7,  1e-8,  1e-9, 1e-10,
    1e-11, 1e-12, 1e-13, 1e-14, 1e-15,  1e-16, 1e-17, 1e-18, 1e-19, 1e-20};
static const double F64_EXP[24] = {
    1.0,  10.0, 100.0, 1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
    1e12, 1e13, 1e14,  1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22, 1e23};
static const int64_t F64_FACT[19] = {1LL,
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

/* falp: (T)(INT_T)((unpacked + base) * FACT[fac]) * FRAC[exp] with unsigned
 * wraparound in the integer part.  This is the generated CPU kernel body for
 * bw < bits(T) (src/alp/falp.cpp:1030-1050: tmp_0 += base_0; tmp_0 *= factor;
 * tmp_int = tmp_0; tmp_dbl = tmp_int; tmp_dbl *= frac10) and the GPU
 * ALPFunctor for every width (src/flsgpu/alp.cuh:40-45).  The reference's
 * CPU full-width kernels (falp.cpp:33293, :42198) deviate -- they multiply
 * the unsigned integer by frac10 and convert the truncated product back --
 * so the full-width case here follows ALPFunctor. */
void orc_falp_f32(const uint32_t *in, float *out, int bw, uint32_t base,
                  int fac, int exp) {
  uint32_t u[VEC];
  orc_unpack_u32(in, u, bw);
  const uint32_t factor = (uint32_t)F32_FACT[fac];
  const float frac = F32_FRAC[exp];
  for (int i = 0; i < VEC; ++i) {
    const uint32_t t = (u[i] + base) * factor;
    const float f = (float)(int32_t)t;
    out[i] = f * frac;
  }
}
void orc_falp_f64(const uint64_t *in, double *out, int bw, uint64_t base,
                  int fac, int exp) {
  uint64_t u[VEC];
  orc_unpack_u64(in, u, bw);
  const uint64_t factor = (uint64_t)F64_FACT[fac];
  const double frac = F64_FRAC[exp];
  for (int i = 0; i < VEC; ++i) {
    const uint64_t t = (u[i] + base) * factor;
    const double d = (double)(int64_t)t;
    out[i] = d * frac;
  }
}

/* ---------------------------------------------------------------------- */
/* Column-level decode: the per-vector loops of src/engine/data.cuh:286-313 */
/* and alp::decode, src/alp/alp-bindings.cu:209-255.                        */
/* ---------------------------------------------------------------------- */
void orc_decode_bp_u32(const uint32_t *packed, const uint8_t *bw,
                       const size_t *offs, size_t n_vecs, uint32_t *out) {
  for (size_t v = 0; v < n_vecs; ++v)
    orc_unpack_u32(packed + offs[v], out + v * VEC, bw[v]);
}
void orc_decode_bp_u64(const uint64_t *packed, const uint8_t *bw,
                       const size_t *offs, size_t n_vecs, uint64_t *out) {
  for (size_t v = 0; v < n_vecs; ++v)
    orc_unpack_u64(packed + offs[v], out + v * VEC, bw[v]);
}
void orc_decode_ffor_u32(const uint32_t *packed, const uint8_t *bw,
                         const size_t *offs, const uint32_t *bases,
                         size_t n_vecs, uint32_t *out) {
  for (size_t v = 0; v < n_vecs; ++v)
    orc_unffor_u32(packed + offs[v], out + v * VEC, bw[v], bases[v]);
}
void orc_decode_ffor_u64(const uint64_t *packed, const uint8_t *bw,
                         const size_t *offs, const uint64_t *bases,
                         size_t n_vecs, uint64_t *out) {
  for (size_t v = 0; v < n_vecs; ++v)
    orc_unffor_u64(packed + offs[v], out + v * VEC, bw[v], bases[v]);
}

/* Exception count of a vector: counts[vi] for ALPColumn; for the extended
 * column, the sum over lanes of (offsets_counts >> 10), exactly as
 * alp::decode(ALPExtendedColumn) reconstructs it (alp-bindings.cu:238-242). */
static size_t vec_exc_count(const uint16_t *counts, const uint16_t *oc,
                            size_t v, int n_lanes) {
  if (counts) return counts[v];
  uint16_t c = 0;
  for (int l = 0; l < n_lanes; ++l) c += (uint16_t)(oc[v * n_lanes + l] >> 10);
  return c;
}

/* decoder::patch_exceptions, src/alp/decoder.hpp:137-145 */
void orc_decode_alp_f32(const uint32_t *packed, const uint8_t *bw,
                        const size_t *offs, const uint32_t *bases,
                        const uint8_t *fac, const uint8_t *exp,
                        const size_t *exc_offs, const float *exc,
                        const uint16_t *pos, const uint16_t *counts,
                        const uint16_t *oc, size_t n_vecs, float *out) {
  for (size_t v = 0; v < n_vecs; ++v) {
    float *o = out + v * VEC;
    orc_falp_f32(packed + offs[v], o, bw[v], bases[v], fac[v], exp[v]);
    const size_t c = vec_exc_count(counts, oc, v, 32);
    for (size_t i = 0; i < c; ++i) o[pos[exc_offs[v] + i]] = exc[exc_offs[v] + i];
  }
}
void orc_decode_alp_f64(const uint64_t *packed, const uint8_t *bw,
                        const size_t *offs, const uint64_t *bases,
                        const uint8_t *fac, const uint8_t *exp,
                        const size_t *exc_offs, const double *exc,
                        const uint16_t *pos, const uint16_t *counts,
                        const uint16_t *oc, size_t n_vecs, double *out) {
  for (size_t v = 0; v < n_vecs; ++v) {
    double *o = out + v * VEC;
    orc_falp_f64(packed + offs[v], o, bw[v], bases[v], fac[v], exp[v]);
    const size_t c = vec_exc_count(counts, oc, v, 16);
    for (size_t i = 0; i < c; ++i) o[pos[exc_offs[v] + i]] = exc[exc_offs[v] + i];
  }
}

/* host::ALPColumn::convert_exceptions_to_lane_divided_format,
 * src/flsgpu/structs.cuh:231-306: exceptions of a vector are regrouped by
 * lane (position % N_LANES), preserving order within a lane, and each lane
 * gets (count << 10) | offset-within-vector in a u16. */
size_t orc_alp_to_extended(int type_bits, const void *exc, const uint16_t *pos,
                           const uint16_t *counts, size_t n_vecs, void *out_exc,
                           uint16_t *out_pos, uint16_t *out_oc) {
  const int N = VEC / type_bits;
  const size_t es = (size_t)type_bits / 8;
  const unsigned char *e = (const unsigned char *)exc;
  unsigned char *oe = (unsigned char *)out_exc;
  size_t base = 0, overflow = 0;
  for (size_t v = 0; v < n_vecs; ++v) {
    const size_t c = counts[v];
    size_t w = 0;
    for (int l = 0; l < N; ++l) {
      size_t lane_count = 0;
      for (size_t i = 0; i < c; ++i) {
        if (pos[base + i] % N != (uint16_t)l) continue;
        memcpy(oe + (base + w) * es, e + (base + i) * es, es);
        out_pos[base + w] = pos[base + i];
        ++w;
        ++lane_count;
      }
      if (lane_count >= 64) ++overflow;
      out_oc[v * N + l] =
          (uint16_t)((lane_count << 10) | ((w - lane_count) & 0xFFFF));
    }
    base += c;
  }
  return overflow;
}

/* ---------------------------------------------------------------------- */
/* ALP encoder, src/alp/encoder.hpp and src/alp/sampler.hpp.               */
/* ---------------------------------------------------------------------- */
#define ENC_UPPER 9223372036854774784.0 /* constants.hpp:18 */
#define ENC_LOWER -9223372036854774784.0

/* sampler::first_level_sample, src/alp/sampler.hpp:11-48, for a rowgroup of
 * whole vectors (config.hpp: ROWGROUP_SIZE 102400, jump 12, 32 samples). */
#define DEFINE_SAMPLER(SUF, PT)                                              \
  static size_t first_level_sample_##SUF(const PT *data, size_t n,         \
                                         PT *smp) {                          \
    const size_t portion = n < 102400 ? n : 102400;                          \
    const size_t nv = (portion + VEC - 1) / VEC;                             \
    size_t si = 0, di = 0;                                                   \
    for (size_t vi = 0; vi < nv; ++vi) {                                     \
      const size_t cur = (n - di) < VEC ? (n - di) : VEC;                    \
      if (vi % 12 != 0) { di += cur; continue; }                             \
      size_t inc = (size_t)ceil((double)cur / 32.0);                         \
      if (inc < 1) inc = 1;                                                  \
      if (cur < 32 && si != 0) { di += cur; continue; }                      \
      for (size_t i = 0; i < cur; i += inc) smp[si++] = data[di + i];        \
      di += cur;                                                             \
    }                                                                        \
    return si;                                                               \
  }
DEFINE_SAMPLER(f64, double)
DEFINE_SAMPLER(f32, float)

static inline int count_bits_u64(uint64_t x) {
  return x == 0 ? 0 : 64 - __builtin_clzll(x);
}
static inline int count_bits_u32(uint32_t x) {
  return x == 0 ? 0 : 32 - __builtin_clz(x);
}

/* encoder::is_impossible_to_encode, encoder.hpp:66-69 */
static inline int impossible_f64(double n) {
  return !isfinite(n) || isnan(n) || n > ENC_UPPER || n < ENC_LOWER ||
         (n == 0.0 && signbit(n));
}
static inline int impossible_f32(float n) {
  return !isfinite(n) || isnan(n) || (double)n > ENC_UPPER ||
         (double)n < ENC_LOWER || (n == 0.0f && signbit(n));
}

/* double -> int64 / float -> int32 truncation with the x86 result for
 * out-of-range inputs ("integer indefinite", INT_MIN), which is what the
 * reference's static_cast compiles to on its CPU. */
static inline int64_t cvtt_f64_s64(double x) {
  if (!(x >= -9223372036854775808.0 && x < 9223372036854775808.0))
    return INT64_MIN;
  return (int64_t)x;
}
static inline int32_t cvtt_f32_s32(float x) {
  if (!(x >= -2147483648.0f && x < 2147483648.0f)) return INT32_MIN;
  return (int32_t)x;
}

/* encoder::encode_value, encoder.hpp:77-84 */
static inline int64_t encode_value_f64(double v, int fac, int exp, int safe) {
  volatile double t = v * F64_EXP[exp];
  t = t * F64_FRAC[fac];
  if (safe && impossible_f64(t)) return cvtt_f64_s64(ENC_UPPER);
  double m = t + 6755399441055744.0; /* MAGIC 0x0018000000000000 */
  m = m - 6755399441055744.0;
  return cvtt_f64_s64(m);
}
static inline int32_t encode_value_f32(float v, int fac, int exp, int safe) {
  volatile float t = v * F32_EXP[exp];
  t = t * F32_FRAC[fac];
  if (safe && impossible_f32(t)) return INT32_MIN;
  float m = t + 12582912.0f;
  m = m - 12582912.0f;
  return cvtt_f32_s32(m);
}
/* decoder::decode_value, decoder.hpp:124-127 */
static inline double decode_value_f64(int64_t e, int fac, int exp) {
  const int64_t p = (int64_t)((uint64_t)e * (uint64_t)F64_FACT[fac]);
  return (double)p * F64_FRAC[exp];
}
static inline float decode_value_f32(int32_t e, int fac, int exp) {
  const int32_t p = (int32_t)((uint32_t)e * (uint32_t)F32_FACT[fac]);
  return (float)p * F32_FRAC[exp];
}

typedef struct {
  int e, f, n;
} combo_t;

/* compare_best_combinations, encoder.hpp:124-128: more occurrences first,
 * then larger exponent, then larger factor. */
static int combo_better(const combo_t *a, const combo_t *b) {
  return (a->n > b->n) || (a->n == b->n && b->e < a->e) ||
         (a->n == b->n && b->e == a->e && b->f < a->f);
}

/* find_top_k_combinations, encoder.hpp:134-230 (generic over PT). */
/* When set, a rowgroup whose best sampled estimate reaches the ALP-RD limit
 * keeps its ALP top-k instead of being rejected (encoder.hpp:208-211 switches
 * such a rowgroup to ALP-RD, which alp::encode turns into an
 * EncodingException, alp-bindings.cu:76-79).  Used to time and size the
 * rowgroup search as an ALP-only encoder on data with ALP-RD rowgroups. */
static int g_rd_as_alp = 0;
void orc_set_rd_as_alp(int on) { g_rd_as_alp = on; }

#define DEFINE_TOPK(SUF, PT, ST, UT, MAXE, EXCBITS, RDLIM, CB)               \
  static int topk_from_sample_##SUF(const PT *smp, size_t n_smp,            \
                                    uint8_t *k_exp, uint8_t *k_fac,         \
                                    uint64_t *best_out) {                   \
    const uint64_t nvs = (uint64_t)ceil((double)((PT)n_smp / (PT)32));     \
    const uint64_t ss = n_smp < 32 ? n_smp : 32;                            \
    combo_t combos[256];                                                    \
    int n_combos = 0;                                                       \
    uint64_t off = 0;                                                       \
    size_t best = ss * (EXCBITS + 16) + ss * EXCBITS;                       \
    for (uint64_t s = 0; s < nvs; ++s) {                                    \
      int fe = 0, ff = 0;                                                   \
      uint64_t sbest = ss * (EXCBITS + 16) + ss * EXCBITS;                  \
      for (int e = MAXE; e >= 0; --e) {                                     \
        for (int f = e; f >= 0; --f) {                                      \
          uint16_t exc = 0, nonexc = 0;                                     \
          ST mx = (ST)((UT)1 << (sizeof(ST) * 8 - 1));                      \
          ST mn = (ST)(((UT)1 << (sizeof(ST) * 8 - 1)) - 1);                \
          for (uint64_t i = 0; i < ss; ++i) {                               \
            const PT a = smp[off + i];                                      \
            const ST enc = encode_value_##SUF(a, f, e, 1);                  \
            const PT dec = decode_value_##SUF(enc, f, e);                   \
            if (dec == a) {                                                 \
              ++nonexc;                                                     \
              if (enc > mx) mx = enc;                                       \
              if (enc < mn) mn = enc;                                       \
            } else {                                                        \
              ++exc;                                                        \
            }                                                               \
          }                                                                 \
          if (nonexc < 2) continue;                                         \
          const uint64_t bits = (uint64_t)CB((UT)mx - (UT)mn);              \
          const uint64_t est = ss * bits + (uint64_t)exc * (EXCBITS + 16);  \
          if (est < sbest || (est == sbest && fe < e) ||                    \
              (est == sbest && fe == e && ff < f)) {                        \
            sbest = est;                                                    \
            fe = e;                                                         \
            ff = f;                                                         \
            if (sbest < best) best = sbest;                                 \
          }                                                                 \
        }                                                                   \
      }                                                                     \
      int found = 0;                                                        \
      for (int c = 0; c < n_combos; ++c)                                    \
        if (combos[c].e == fe && combos[c].f == ff) {                       \
          combos[c].n++;                                                    \
          found = 1;                                                        \
        }                                                                   \
      if (!found) {                                                         \
        combos[n_combos].e = fe;                                            \
        combos[n_combos].f = ff;                                            \
        combos[n_combos].n = 1;                                             \
        ++n_combos;                                                         \
      }                                                                     \
      off += ss;                                                            \
    }                                                                       \
    if (best_out) *best_out = best;                                         \
    if (best >= RDLIM && !g_rd_as_alp) return -1;                          \
    /* selection sort with the reference's strict total order */            \
    for (int i = 0; i < n_combos; ++i)                                      \
      for (int j = i + 1; j < n_combos; ++j)                                \
        if (combo_better(&combos[j], &combos[i])) {                         \
          combo_t t = combos[i];                                            \
          combos[i] = combos[j];                                            \
          combos[j] = t;                                                    \
        }                                                                   \
    const int k = n_combos < 5 ? n_combos : 5;                              \
    for (int i = 0; i < k; ++i) {                                           \
      k_exp[i] = (uint8_t)combos[i].e;                                      \
      k_fac[i] = (uint8_t)combos[i].f;                                      \
    }                                                                       \
    return k;                                                               \
  }

DEFINE_TOPK(f64, double, int64_t, uint64_t, 18, 64, 48 * 32, count_bits_u64)
DEFINE_TOPK(f32, float, int32_t, uint32_t, 10, 32, 22 * 32, count_bits_u32)

int orc_alp_rowgroup_topk_f64(const double *rg, size_t n, uint8_t *ke,
                              uint8_t *kf) {
  double *smp = (double *)malloc(sizeof(double) * (n + 32));
  const size_t ns = first_level_sample_f64(rg, n, smp);
  const int k = topk_from_sample_f64(smp, ns, ke, kf, NULL);
  free(smp);
  return k;
}
int orc_alp_rowgroup_topk_f32(const float *rg, size_t n, uint8_t *ke,
                              uint8_t *kf) {
  float *smp = (float *)malloc(sizeof(float) * (n + 32));
  const size_t ns = first_level_sample_f32(rg, n, smp);
  const int k = topk_from_sample_f32(smp, ns, ke, kf, NULL);
  free(smp);
  return k;
}

int orc_alp_vector_best_f64(const double *vec, uint64_t *est_bits) {
  double smp[32];
  for (int i = 0; i < 32; ++i) smp[i] = vec[i * 32];
  uint8_t ke[5], kf[5];
  uint64_t best = 0;
  /* one sampled vector: the single combination found is the winner */
  const int k = topk_from_sample_f64(smp, 32, ke, kf, &best);
  if (est_bits) *est_bits = best;
  if (k <= 0) return -1;
  return ke[0] * 32 + kf[0];
}

int orc_alp_vector_best_f32(const float *vec, uint64_t *est_bits) {
  float smp[32];
  for (int i = 0; i < 32; ++i) smp[i] = vec[i * 32];
  uint8_t ke[5], kf[5];
  uint64_t best = 0;
  const int saved = g_rd_as_alp;
  g_rd_as_alp = 1; /* the pair is wanted even where ALP-RD would be chosen */
  const int k = topk_from_sample_f32(smp, 32, ke, kf, &best);
  g_rd_as_alp = saved;
  if (est_bits) *est_bits = best;
  if (k <= 0) return -1;
  return ke[0] * 32 + kf[0];
}

/* find_best_exponent_factor_from_combinations, encoder.hpp:237-300 */
#define DEFINE_CHOOSE(SUF, PT, ST, UT, EXCBITS, CB)                          \
  static void choose_##SUF(const PT *vec, int k, const uint8_t *ke,         \
                           const uint8_t *kf, uint8_t *exp, uint8_t *fac) { \
    int fe = 0, ff = 0, worse = 0;                                          \
    uint64_t best = 0;                                                      \
    for (int c = 0; c < k; ++c) {                                           \
      const int e = ke[c], f = kf[c];                                       \
      uint32_t exc = 0;                                                     \
      ST mx = (ST)((UT)1 << (sizeof(ST) * 8 - 1));                          \
      ST mn = (ST)(((UT)1 << (sizeof(ST) * 8 - 1)) - 1);                    \
      for (int i = 0; i < VEC; i += 32) {                                   \
        const PT a = vec[i];                                                \
        const ST enc = encode_value_##SUF(a, f, e, 1);                      \
        const PT dec = decode_value_##SUF(enc, f, e);                       \
        if (dec == a) {                                                     \
          if (enc > mx) mx = enc;                                           \
          if (enc < mn) mn = enc;                                           \
        } else {                                                            \
          ++exc;                                                            \
        }                                                                   \
      }                                                                     \
      const uint64_t est =                                                  \
          32 * (uint64_t)CB((UT)mx - (UT)mn) + (uint64_t)exc * (EXCBITS + 16); \
      if (c == 0) {                                                         \
        best = est;                                                         \
        ff = f;                                                             \
        fe = e;                                                             \
        continue;                                                           \
      }                                                                     \
      if (est >= best) {                                                    \
        if (++worse == 2) break;                                            \
        continue;                                                           \
      }                                                                     \
      best = est;                                                           \
      ff = f;                                                               \
      fe = e;                                                               \
      worse = 0;                                                            \
    }                                                                       \
    *exp = (uint8_t)fe;                                                     \
    *fac = (uint8_t)ff;                                                     \
  }
DEFINE_CHOOSE(f64, double, int64_t, uint64_t, 64, count_bits_u64)
DEFINE_CHOOSE(f32, float, int32_t, uint32_t, 32, count_bits_u32)

void orc_alp_vector_choose_f64(const double *vec, int k, const uint8_t *ke,
                               const uint8_t *kf, uint8_t *exp, uint8_t *fac) {
  if (k > 1) {
    choose_f64(vec, k, ke, kf, exp, fac);
  } else {
    *exp = ke[0];
    *fac = kf[0];
  }
}

/* encoder::encode_simdized, encoder.hpp:302-379.  Special values (NaN,
 * +-inf, -0.0) are replaced by ENCODING_UPPER_LIMIT before the trial
 * encode; positions whose round trip differs are exceptions storing the
 * original value; their integer is replaced by the integer of the first
 * non-exception position (the INDEX_ARR scan at :361-367, which yields 0
 * when every position, or every position but the last, is an exception). */
#define DEFINE_ENCVEC(SUF, PT, ST, UT, SIGNMASK, EXPMASK, NEGZERO)           \
  static int encode_vector_##SUF(const PT *vec, int e, int f, ST *enc,      \
                                 PT *exc, uint16_t *pos) {                  \
    int n_exc = 0, first_ok = -1;                                           \
    for (int i = 0; i < VEC; ++i) {                                         \
      UT bits;                                                              \
      memcpy(&bits, &vec[i], sizeof(UT));                                   \
      const int special = ((bits & SIGNMASK) >= EXPMASK) || bits == NEGZERO; \
      const PT a = special ? (PT)ENC_UPPER : vec[i];                        \
      enc[i] = encode_value_##SUF(a, f, e, 0);                              \
      const PT dec = decode_value_##SUF(enc[i], f, e);                      \
      if (dec != a) {                                                       \
        pos[n_exc] = (uint16_t)i;                                           \
        exc[n_exc] = vec[i];                                                \
        ++n_exc;                                                            \
      } else if (first_ok < 0) {                                            \
        first_ok = i;                                                       \
      }                                                                     \
    }                                                                       \
    ST fill = 0;                                                            \
    if (first_ok >= 0 && !(first_ok == VEC - 1 && n_exc == VEC - 1))        \
      fill = enc[first_ok];                                                 \
    for (int j = 0; j < n_exc; ++j) enc[pos[j]] = fill;                     \
    return n_exc;                                                           \
  }
DEFINE_ENCVEC(f64, double, int64_t, uint64_t, 0x7FFFFFFFFFFFFFFFULL,
              0x7FF0000000000000ULL, 0x8000000000000000ULL)
DEFINE_ENCVEC(f32, float, int32_t, uint32_t, 0x7FFFFFFFU, 0x7F800000U,
              0x80000000U)

int orc_alp_encode_vector_f64(const double *vec, int exp, int fac,
                              int64_t *encoded, double *exc, uint16_t *pos) {
  return encode_vector_f64(vec, exp, fac, encoded, exc, pos);
}
int orc_alp_encode_vector_f32(const float *vec, int exp, int fac, int32_t *encoded, float *exc,
                              uint16_t *pos) {
  return encode_vector_f32(vec, exp, fac, encoded, exc, pos);
}

/* alp::encode, src/alp/alp-bindings.cu:84-206: per vector, second-level
 * choice + encode_simdized, then analyze_ffor (encoder.hpp:104-115: base =
 * signed min, bw = bits(max - min)) and fls::ffor.  Byte accounting as
 * alp-bindings.cu:19-43. */
#define DEFINE_ENCODE(SUF, PT, ST, UT, NL)                                   \
  int orc_alp_encode_##SUF(const PT *in, size_t n_vecs, size_t rg_vecs,     \
                           UT *packed, uint8_t *bw, size_t *offs,           \
                           UT *bases, uint8_t *fac, uint8_t *exp,           \
                           size_t *exc_offs, PT *exc, uint16_t *pos,        \
                           uint16_t *counts, orc_alp_encode_info *info) {   \
    uint8_t ke[5], kf[5];                                                   \
    int k = 0;                                                              \
    size_t n_packed = 0, n_exc = 0, body = 0;                               \
    PT *smp = (PT *)malloc(sizeof(PT) * 102400 + 32 * sizeof(PT));          \
    ST enc[VEC];                                                            \
    memset(info, 0, sizeof(*info));                                         \
    for (size_t v = 0; v < n_vecs; ++v) {                                   \
      const int new_rg = (v == 0) || (rg_vecs != 0 && v % rg_vecs == 0);    \
      if (new_rg) {                                                         \
        const size_t rem = (n_vecs - v) * VEC;                              \
        const size_t ns = first_level_sample_##SUF(in + v * VEC, rem, smp); \
        k = topk_from_sample_##SUF(smp, ns, ke, kf, NULL);                  \
        if (k < 0) {                                                        \
          info->rd_rowgroup = rg_vecs ? v / rg_vecs : 0;                    \
          free(smp);                                                        \
          return 1;                                                         \
        }                                                                   \
      }                                                                     \
      const PT *vec = in + v * VEC;                                         \
      uint8_t e, f;                                                         \
      if (k > 1) {                                                          \
        choose_##SUF(vec, k, ke, kf, &e, &f);                               \
      } else {                                                              \
        e = ke[0];                                                          \
        f = kf[0];                                                          \
      }                                                                     \
      const int c = encode_vector_##SUF(vec, e, f, enc, exc + n_exc,        \
                                        pos + n_exc);                       \
      ST mn = enc[0], mx = enc[0];                                          \
      for (int i = 1; i < VEC; ++i) {                                       \
        if (enc[i] < mn) mn = enc[i];                                       \
        if (enc[i] > mx) mx = enc[i];                                       \
      }                                                                     \
      const int w = (sizeof(UT) == 8) ? count_bits_u64((UT)mx - (UT)mn)     \
                                      : count_bits_u32((UT)mx - (UT)mn);    \
      bw[v] = (uint8_t)w;                                                   \
      bases[v] = (UT)mn;                                                    \
      orc_ffor_u##NL((const UT *)enc, packed + n_packed, w, (UT)mn);        \
      offs[v] = n_packed;                                                   \
      n_packed += (size_t)w * (1024 / NL);                                  \
      fac[v] = f;                                                           \
      exp[v] = e;                                                           \
      exc_offs[v] = n_exc;                                                  \
      counts[v] = (uint16_t)c;                                              \
      n_exc += (size_t)c;                                                   \
      body += (size_t)w * (1024 / NL) * sizeof(PT) +                        \
              (size_t)c * (sizeof(PT) + 2);                                 \
    }                                                                       \
    free(smp);                                                              \
    info->n_packed = n_packed;                                              \
    info->n_exceptions = n_exc;                                             \
    info->compressed_bytes = body + n_vecs * (3 + sizeof(PT));              \
    info->compressed_bytes_extended =                                       \
        body + n_vecs * (3 + sizeof(PT) + 2 * (1024 / NL));                 \
    return 0;                                                               \
  }
DEFINE_ENCODE(f64, double, int64_t, uint64_t, 64)
DEFINE_ENCODE(f32, float, int32_t, uint32_t, 32)

/* ---------------------------------------------------------------------- */
/* ALP-RD, src/alp/rd.hpp.                                                  */
/* ---------------------------------------------------------------------- */
typedef struct {
  uint64_t key;
  int32_t n;
} lp_t;

/* build_left_parts_dictionary, rd.hpp:28-81.  The reference orders left
 * parts by occurrence count through an unordered_map + std::sort, so ties
 * land in an implementation-defined order; here ties are broken by smaller
 * left part first.  The estimated size, and therefore the chosen cut, is
 * independent of the tie order. */
static double rd_build_dict(const uint64_t *bits, size_t n, int rbw, int tb,
                            orc_rd_state *st) {
  lp_t *lp = (lp_t *)malloc(sizeof(lp_t) * (n + 1));
  size_t m = 0;
  for (size_t i = 0; i < n; ++i) {
    const uint64_t key = bits[i] >> rbw;
    size_t j = 0;
    for (; j < m; ++j)
      if (lp[j].key == key) break;
    if (j == m) {
      lp[m].key = key;
      lp[m].n = 0;
      ++m;
    }
    lp[j].n++;
  }
  for (size_t i = 0; i < m; ++i)
    for (size_t j = i + 1; j < m; ++j)
      if (lp[j].n > lp[i].n || (lp[j].n == lp[i].n && lp[j].key < lp[i].key)) {
        lp_t t = lp[i];
        lp[i] = lp[j];
        lp[j] = t;
      }
  uint32_t exc = 0;
  for (size_t i = 8; i < m; ++i) exc += (uint32_t)lp[i].n;
  const int dsize = m < 8 ? (int)m : 8;
  int lbw = (int)ceil(log2((double)dsize));
  if (lbw < 1) lbw = 1;
  if (st) {
    memset(st, 0, sizeof(*st));
    for (int i = 0; i < dsize; ++i) st->dict[i] = (uint16_t)lp[i].key;
    st->left_bw = (uint8_t)lbw;
    st->right_bw = (uint8_t)rbw;
    st->dict_size = (uint8_t)dsize;
  }
  free(lp);
  (void)tb;
  /* estimate_compression_size, rd.hpp:18-25 */
  return (double)rbw + (double)lbw + (double)exc * (16 + 16) / (double)n;
}

/* find_best_dictionary, rd.hpp:83-98: cut 1..16 bits from the top. */
static void rd_init_bits(const uint64_t *bits, size_t n, int tb,
                         orc_rd_state *st) {
  int best_rbw = 0;
  double best = 1.7976931348623157e308;
  for (int i = 1; i <= 16; ++i) {
    const int cand = tb - i;
    const double est = rd_build_dict(bits, n, cand, tb, NULL);
    if (est < best) {
      best_rbw = cand;
      best = est;
    }
  }
  rd_build_dict(bits, n, best_rbw, tb, st);
}

void orc_rd_init_f64(const double *rg, size_t n, orc_rd_state *st) {
  double *smp = (double *)malloc(sizeof(double) * 102400 + 256);
  const size_t ns = first_level_sample_f64(rg, n, smp);
  uint64_t *bits = (uint64_t *)malloc(sizeof(uint64_t) * (ns + 1));
  memcpy(bits, smp, sizeof(uint64_t) * ns);
  rd_init_bits(bits, ns, 64, st);
  free(bits);
  free(smp);
}
void orc_rd_init_f32(const float *rg, size_t n, orc_rd_state *st) {
  float *smp = (float *)malloc(sizeof(float) * 102400 + 256);
  const size_t ns = first_level_sample_f32(rg, n, smp);
  uint64_t *bits = (uint64_t *)malloc(sizeof(uint64_t) * (ns + 1));
  for (size_t i = 0; i < ns; ++i) {
    uint32_t b;
    memcpy(&b, &smp[i], 4);
    bits[i] = b;
  }
  rd_init_bits(bits, ns, 32, st);
  free(bits);
  free(smp);
}

/* rd_encoder::encode, rd.hpp:103-140 */
#define DEFINE_RD_ENC(SUF, PT, UT)                                            \
  int orc_rd_encode_vector_##SUF(const PT *vec, const orc_rd_state *st,      \
                                 UT *right, uint16_t *left_idx,             \
                                 uint16_t *exc, uint16_t *pos) {            \
    int n_exc = 0;                                                          \
    for (int i = 0; i < VEC; ++i) {                                         \
      UT b;                                                                 \
      memcpy(&b, &vec[i], sizeof(UT));                                      \
      right[i] = (UT)(b & (UT)(((uint64_t)1 << st->right_bw) - 1));         \
      const uint16_t left = (uint16_t)(b >> st->right_bw);                  \
      int idx = st->dict_size;                                              \
      for (int d = 0; d < st->dict_size; ++d)                               \
        if (st->dict[d] == left) {                                          \
          idx = d;                                                          \
          break;                                                            \
        }                                                                   \
      left_idx[i] = (uint16_t)idx;                                          \
      if (idx >= st->dict_size) {                                           \
        exc[n_exc] = left;                                                  \
        pos[n_exc] = (uint16_t)i;                                           \
        ++n_exc;                                                            \
      }                                                                     \
    }                                                                       \
    return n_exc;                                                           \
  }
DEFINE_RD_ENC(f64, double, uint64_t)
DEFINE_RD_ENC(f32, float, uint32_t)

/* rd_encoder::decode, rd.hpp:146-172.  A dictionary index at or beyond
 * the dictionary (only ever at exception positions, which are patched
 * afterwards) reads entry 7 here instead of the reference's out-of-bounds
 * neighbour. */
#define DEFINE_RD_DEC(SUF, PT, UT)                                            \
  void orc_rd_decode_vector_##SUF(const UT *right, const uint16_t *left_idx, \
                                  const uint16_t *dict, int rbw,            \
                                  const uint16_t *exc, const uint16_t *pos, \
                                  int n_exc, PT *out) {                     \
    UT *o = (UT *)out;                                                      \
    for (int i = 0; i < VEC; ++i) {                                         \
      const uint16_t li = left_idx[i] < 8 ? left_idx[i] : 7;                \
      o[i] = ((UT)dict[li] << rbw) | right[i];                              \
    }                                                                       \
    for (int i = 0; i < n_exc; ++i)                                         \
      o[pos[i]] = ((UT)exc[i] << rbw) | right[pos[i]];                      \
  }
DEFINE_RD_DEC(f64, double, uint64_t)
DEFINE_RD_DEC(f32, float, uint32_t)

#define DEFINE_RD_COL(SUF, PT, UT, TB)                                        \
  void orc_decode_rd_##SUF(const UT *rp, const size_t *ro, const uint8_t *rb, \
                           const uint16_t *lp, const size_t *lo,            \
                           const uint8_t *lb, const uint16_t *dicts,        \
                           const uint32_t *di, const size_t *eo,            \
                           const uint16_t *exc, const uint16_t *pos,        \
                           const uint16_t *counts, size_t n_vecs, PT *out) {\
    UT right[VEC];                                                          \
    uint16_t left[VEC];                                                     \
    for (size_t v = 0; v < n_vecs; ++v) {                                   \
      orc_unpack_u##TB(rp + ro[v], right, rb[v]);                           \
      orc_unpack_u16(lp + lo[v], left, lb[v]);                              \
      orc_rd_decode_vector_##SUF(right, left, dicts + 8 * (size_t)di[v],    \
                                 rb[v], exc + eo[v], pos + eo[v],           \
                                 counts[v], out + v * VEC);                 \
    }                                                                       \
  }
DEFINE_RD_COL(f64, double, uint64_t, 64)
DEFINE_RD_COL(f32, float, uint32_t, 32)

/* ---------------------------------------------------------------------- */
/* Fixed-order reductions used by the fused kernels.                        */
/* ---------------------------------------------------------------------- */
/* Thread t of a 32-thread warp owns lane t % N and, for 64-bit types,
 * value half t / 16 (values 32*h .. 32*h+31 of the lane).  It adds its 32
 * values in ascending order starting from +0.0; the warp then combines by
 * butterfly (p[t] = p[t] + p[t ^ s], s = 16, 8, 4, 2, 1) and thread 0's
 * value is the vector partial.  Vector partials are combined pairwise with
 * doubling stride: p[i] += p[i + s] for i % 2s == 0, s = 1, 2, 4, ... */
static double warp_tree_f64(double p[32]) {
  for (int s = 16; s >= 1; s >>= 1) {
    double q[32];
    for (int t = 0; t < 32; ++t) q[t] = p[t] + p[t ^ s];
    memcpy(p, q, sizeof(q));
  }
  return p[0];
}
static float warp_tree_f32(float p[32]) {
  for (int s = 16; s >= 1; s >>= 1) {
    float q[32];
    for (int t = 0; t < 32; ++t) q[t] = p[t] + p[t ^ s];
    memcpy(p, q, sizeof(q));
  }
  return p[0];
}
static double pairwise_f64(double *p, size_t n) {
  if (n == 0) return 0.0;
  for (size_t s = 1; s < n; s <<= 1)
    for (size_t i = 0; i + s < n; i += 2 * s) p[i] = p[i] + p[i + s];
  return p[0];
}

double orc_tree_sum_masked_f64(const double *values, const uint32_t *keys,
                               uint32_t thr, size_t n_vecs) {
  double *part = (double *)malloc(sizeof(double) * (n_vecs + 1));
  for (size_t v = 0; v < n_vecs; ++v) {
    const double *x = values + v * VEC;
    const uint32_t *kk = keys ? keys + v * VEC : NULL;
    double p[32];
    for (int t = 0; t < 32; ++t) {
      const int l = t & 15, h = t >> 4;
      double acc = 0.0;
      for (int k = 0; k < 32; ++k) {
        const size_t idx = (size_t)l + 16 * (size_t)(32 * h + k);
        if (!kk || kk[idx] < thr) acc = acc + x[idx];
      }
      p[t] = acc;
    }
    part[v] = warp_tree_f64(p);
  }
  const double r = pairwise_f64(part, n_vecs);
  free(part);
  return r;
}
double orc_tree_sum_f64(const double *values, size_t n_vecs) {
  return orc_tree_sum_masked_f64(values, NULL, 0, n_vecs);
}
float orc_tree_sum_f32(const float *values, size_t n_vecs) {
  float *part = (float *)malloc(sizeof(float) * (n_vecs + 1));
  for (size_t v = 0; v < n_vecs; ++v) {
    const float *x = values + v * VEC;
    float p[32];
    for (int t = 0; t < 32; ++t) {
      float acc = 0.0f;
      for (int k = 0; k < 32; ++k) acc = acc + x[t + 32 * k];
      p[t] = acc;
    }
    part[v] = warp_tree_f32(p);
  }
  float r = 0.0f;
  if (n_vecs) {
    for (size_t s = 1; s < n_vecs; s <<= 1)
      for (size_t i = 0; i + s < n_vecs; i += 2 * s) part[i] = part[i] + part[i + s];
    r = part[0];
  }
  free(part);
  return r;
}
uint64_t orc_sum_u32(const uint32_t *values, size_t n) {
  uint64_t s = 0;
  for (size_t i = 0; i < n; ++i) s += values[i];
  return s;
}
uint64_t orc_sum_u64(const uint64_t *values, size_t n) {
  uint64_t s = 0;
  for (size_t i = 0; i < n; ++i) s += values[i];
  return s;
}

static int cmp_u32(const void *a, const void *b) {
  const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return (x > y) - (x < y);
}
uint32_t orc_median_u32(const uint32_t *values, size_t n) {
  if (n == 0) return 0;
  uint32_t *c = (uint32_t *)malloc(sizeof(uint32_t) * n);
  memcpy(c, values, sizeof(uint32_t) * n);
  qsort(c, n, sizeof(uint32_t), cmp_u32);
  const uint32_t m = c[(n - 1) / 2];
  free(c);
  return m;
}
