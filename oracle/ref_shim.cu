// ref_shim.cu -- TEST INFRASTRUCTURE ONLY.
//
// extern "C" entry points over the reference's own CPU codecs, compiled
// together with the reference's unmodified sources (src/fls/*.cpp,
// src/alp/falp.cpp, src/alp/alp-bindings.cu) by oracle/build_ref.sh into
// oracle/_ref/libflsref.so.  Used to pin the oracle restatement (golden
// vectors, tests/golden/gen_golden.py) and as the timed CPU baseline of
// bench.py.  Host code only: nothing here launches a kernel.
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "src/alp/alp-bindings.cuh"
#include "src/alp/decoder.hpp"
#include "src/alp/encoder.hpp"
#include "src/alp/falp.hpp"
#include "src/alp/rd.hpp"
#include "src/fls/fls-bindings.hpp"


extern "C" void ref_pack_u16(const uint16_t *in, uint16_t *out, int bw) { fls::pack(in, out, (uint8_t)bw); }
extern "C" void ref_pack_u32(const uint32_t *in, uint32_t *out, int bw) { fls::pack(in, out, (uint8_t)bw); }
extern "C" void ref_pack_u64(const uint64_t *in, uint64_t *out, int bw) { fls::pack(in, out, (uint8_t)bw); }
extern "C" void ref_unpack_u16(const uint16_t *in, uint16_t *out, int bw) { fls::unpack(in, out, (uint8_t)bw); }
extern "C" void ref_unpack_u32(const uint32_t *in, uint32_t *out, int bw) { fls::unpack(in, out, (uint8_t)bw); }
extern "C" void ref_unpack_u64(const uint64_t *in, uint64_t *out, int bw) { fls::unpack(in, out, (uint8_t)bw); }
extern "C" void ref_pack_u8(const uint8_t *in, uint8_t *out, int bw) { fls::pack(in, out, (uint8_t)bw); }
extern "C" void ref_unpack_u8(const uint8_t *in, uint8_t *out, int bw) { fls::unpack(in, out, (uint8_t)bw); }
extern "C" void ref_ffor_u8(const uint8_t *in, uint8_t *out, int bw, uint8_t base) { fls::ffor(in, out, (uint8_t)bw, &base); }
extern "C" void ref_ffor_u16(const uint16_t *in, uint16_t *out, int bw, uint16_t base) { fls::ffor(in, out, (uint8_t)bw, &base); }
extern "C" void ref_unffor_u8(const uint8_t *in, uint8_t *out, int bw, uint8_t base) { fls::unffor(in, out, (uint8_t)bw, &base); }
extern "C" void ref_unffor_u16(const uint16_t *in, uint16_t *out, int bw, uint16_t base) { fls::unffor(in, out, (uint8_t)bw, &base); }
extern "C" void ref_ffor_u32(const uint32_t *in, uint32_t *out, int bw, uint32_t base) { fls::ffor(in, out, (uint8_t)bw, &base); }
extern "C" void ref_ffor_u64(const uint64_t *in, uint64_t *out, int bw, uint64_t base) { fls::ffor(in, out, (uint8_t)bw, &base); }
extern "C" void ref_unffor_u32(const uint32_t *in, uint32_t *out, int bw, uint32_t base) { fls::unffor(in, out, (uint8_t)bw, &base); }
extern "C" void ref_unffor_u64(const uint64_t *in, uint64_t *out, int bw, uint64_t base) { fls::unffor(in, out, (uint8_t)bw, &base); }

extern "C" void ref_falp_f32(const uint32_t *in, float *out, int bw, uint32_t base, int fac, int exp) {
  generated::falp::fallback::scalar::falp(in, out, (uint8_t)bw, &base, (uint8_t)fac, (uint8_t)exp);
}
extern "C" void ref_falp_f64(const uint64_t *in, double *out, int bw, uint64_t base, int fac, int exp) {
  generated::falp::fallback::scalar::falp(in, out, (uint8_t)bw, &base, (uint8_t)fac, (uint8_t)exp);
}

// Vector loops of src/engine/data.cuh:286-313 over [v0, v1).
extern "C" void ref_decode_ffor_u32(const uint32_t *packed, const uint8_t *bw, const size_t *offs,
                         const uint32_t *bases, size_t v0, size_t v1, uint32_t *out) {
  for (size_t v = v0; v < v1; ++v) fls::unffor(packed + offs[v], out + v * 1024, bw[v], &bases[v]);
}
extern "C" void ref_decode_ffor_u64(const uint64_t *packed, const uint8_t *bw, const size_t *offs,
                         const uint64_t *bases, size_t v0, size_t v1, uint64_t *out) {
  for (size_t v = v0; v < v1; ++v) fls::unffor(packed + offs[v], out + v * 1024, bw[v], &bases[v]);
}

template <typename T, typename UT>
static flsgpu::host::ALPColumn<T> make_column(const UT *packed, size_t n_packed, const uint8_t *bw,
                                             const size_t *offs, const UT *bases, const uint8_t *fac,
                                             const uint8_t *exp, const size_t *exc_offs, const T *exc,
                                             const uint16_t *pos, const uint16_t *counts,
                                             size_t n_vecs, size_t n_exc) {
  flsgpu::host::ALPColumn<T> c{};
  c.ffor.bp.n_values = n_vecs * 1024;
  c.ffor.bp.n_packed_values = n_packed;
  c.ffor.bp.packed_array = const_cast<UT *>(packed);
  c.ffor.bp.bit_widths = const_cast<uint8_t *>(bw);
  c.ffor.bp.vector_offsets = const_cast<size_t *>(offs);
  c.ffor.bases = const_cast<UT *>(bases);
  c.factor_indices = const_cast<uint8_t *>(fac);
  c.fraction_indices = const_cast<uint8_t *>(exp);
  c.n_exceptions = n_exc;
  c.exceptions_offsets = const_cast<size_t *>(exc_offs);
  c.exceptions = const_cast<T *>(exc);
  c.positions = const_cast<uint16_t *>(pos);
  c.counts = const_cast<uint16_t *>(counts);
  return c;
}

// alp::decode(ALPColumn), src/alp/alp-bindings.cu:209-227, on [v0, v1).
extern "C" void ref_decode_alp_f64(const uint64_t *packed, const uint8_t *bw, const size_t *offs,
                        const uint64_t *bases, const uint8_t *fac, const uint8_t *exp,
                        const size_t *exc_offs, const double *exc, const uint16_t *pos,
                        const uint16_t *counts, size_t v0, size_t v1, double *out) {
  auto c = make_column<double, uint64_t>(packed, 0, bw + v0, offs + v0, bases + v0, fac + v0,
                                         exp + v0, exc_offs + v0, exc, pos, counts + v0,
                                         v1 - v0, 0);
  alp::decode(c, out + v0 * 1024);
}
extern "C" void ref_decode_alp_f32(const uint32_t *packed, const uint8_t *bw, const size_t *offs,
                        const uint32_t *bases, const uint8_t *fac, const uint8_t *exp,
                        const size_t *exc_offs, const float *exc, const uint16_t *pos,
                        const uint16_t *counts, size_t v0, size_t v1, float *out) {
  auto c = make_column<float, uint32_t>(packed, 0, bw + v0, offs + v0, bases + v0, fac + v0,
                                        exp + v0, exc_offs + v0, exc, pos, counts + v0,
                                        v1 - v0, 0);
  alp::decode(c, out + v0 * 1024);
}

// alp::decode(ALPExtendedColumn), alp-bindings.cu:230-255.
extern "C" void ref_decode_alpx_f64(const uint64_t *packed, const uint8_t *bw, const size_t *offs,
                         const uint64_t *bases, const uint8_t *fac, const uint8_t *exp,
                         const size_t *exc_offs, const double *exc, const uint16_t *pos,
                         const uint16_t *offsets_counts, size_t n_vecs, double *out) {
  flsgpu::host::ALPExtendedColumn<double> c{};
  c.ffor.bp.n_values = n_vecs * 1024;
  c.ffor.bp.packed_array = const_cast<uint64_t *>(packed);
  c.ffor.bp.bit_widths = const_cast<uint8_t *>(bw);
  c.ffor.bp.vector_offsets = const_cast<size_t *>(offs);
  c.ffor.bases = const_cast<uint64_t *>(bases);
  c.factor_indices = const_cast<uint8_t *>(fac);
  c.fraction_indices = const_cast<uint8_t *>(exp);
  c.exceptions_offsets = const_cast<size_t *>(exc_offs);
  c.exceptions = const_cast<double *>(exc);
  c.positions = const_cast<uint16_t *>(pos);
  c.offsets_counts = const_cast<uint16_t *>(offsets_counts);
  alp::decode(c, out);
}
extern "C" void ref_decode_alpx_f32(const uint32_t *packed, const uint8_t *bw, const size_t *offs,
                         const uint32_t *bases, const uint8_t *fac, const uint8_t *exp,
                         const size_t *exc_offs, const float *exc, const uint16_t *pos,
                         const uint16_t *offsets_counts, size_t n_vecs, float *out) {
  flsgpu::host::ALPExtendedColumn<float> c{};
  c.ffor.bp.n_values = n_vecs * 1024;
  c.ffor.bp.packed_array = const_cast<uint32_t *>(packed);
  c.ffor.bp.bit_widths = const_cast<uint8_t *>(bw);
  c.ffor.bp.vector_offsets = const_cast<size_t *>(offs);
  c.ffor.bases = const_cast<uint32_t *>(bases);
  c.factor_indices = const_cast<uint8_t *>(fac);
  c.fraction_indices = const_cast<uint8_t *>(exp);
  c.exceptions_offsets = const_cast<size_t *>(exc_offs);
  c.exceptions = const_cast<float *>(exc);
  c.positions = const_cast<uint16_t *>(pos);
  c.offsets_counts = const_cast<uint16_t *>(offsets_counts);
  alp::decode(c, out);
}

// host::ALPColumn::convert_exceptions_to_lane_divided_format, structs.cuh:231.
extern "C" void ref_alp_to_extended_f64(const double *exc, const uint16_t *pos, const uint16_t *counts,
                             size_t n_vecs, size_t n_exc, double *out_exc, uint16_t *out_pos,
                             uint16_t *out_oc) {
  flsgpu::host::ALPColumn<double> c{};
  c.ffor.bp.n_values = n_vecs * 1024;
  c.n_exceptions = n_exc;
  c.exceptions = const_cast<double *>(exc);
  c.positions = const_cast<uint16_t *>(pos);
  c.counts = const_cast<uint16_t *>(counts);
  auto [e, p, oc] = c.convert_exceptions_to_lane_divided_format();
  std::memcpy(out_exc, e, sizeof(double) * n_exc);
  std::memcpy(out_pos, p, sizeof(uint16_t) * n_exc);
  std::memcpy(out_oc, oc, sizeof(uint16_t) * n_vecs * 16);
  free(e);
  free(p);
  free(oc);
}
extern "C" void ref_alp_to_extended_f32(const float *exc, const uint16_t *pos, const uint16_t *counts,
                             size_t n_vecs, size_t n_exc, float *out_exc, uint16_t *out_pos,
                             uint16_t *out_oc) {
  flsgpu::host::ALPColumn<float> c{};
  c.ffor.bp.n_values = n_vecs * 1024;
  c.n_exceptions = n_exc;
  c.exceptions = const_cast<float *>(exc);
  c.positions = const_cast<uint16_t *>(pos);
  c.counts = const_cast<uint16_t *>(counts);
  auto [e, p, oc] = c.convert_exceptions_to_lane_divided_format();
  std::memcpy(out_exc, e, sizeof(float) * n_exc);
  std::memcpy(out_pos, p, sizeof(uint16_t) * n_exc);
  std::memcpy(out_oc, oc, sizeof(uint16_t) * n_vecs * 32);
  free(e);
  free(p);
  free(oc);
}

// alp::encode, src/alp/alp-bindings.cu:84-206.  Returns 0, or 1 on
// alp::EncodingException (sampling chose ALP-RD).
template <typename T, typename UT>
static int encode_impl(const T *in, size_t n_values, UT *packed, uint8_t *bw, size_t *offs,
                       UT *bases, uint8_t *fac, uint8_t *exp, size_t *exc_offs, T *exc,
                       uint16_t *pos, uint16_t *counts, size_t *sizes) {
  try {
    auto c = alp::encode<T>(in, n_values, false);
    const size_t n_vecs = c.get_n_vecs();
    std::memcpy(packed, c.ffor.bp.packed_array, sizeof(UT) * c.ffor.bp.n_packed_values);
    std::memcpy(bw, c.ffor.bp.bit_widths, n_vecs);
    std::memcpy(offs, c.ffor.bp.vector_offsets, sizeof(size_t) * n_vecs);
    std::memcpy(bases, c.ffor.bases, sizeof(UT) * n_vecs);
    std::memcpy(fac, c.factor_indices, n_vecs);
    std::memcpy(exp, c.fraction_indices, n_vecs);
    std::memcpy(exc_offs, c.exceptions_offsets, sizeof(size_t) * n_vecs);
    std::memcpy(exc, c.exceptions, sizeof(T) * c.n_exceptions);
    std::memcpy(pos, c.positions, sizeof(uint16_t) * c.n_exceptions);
    std::memcpy(counts, c.counts, sizeof(uint16_t) * n_vecs);
    sizes[0] = c.ffor.bp.n_packed_values;
    sizes[1] = c.n_exceptions;
    sizes[2] = c.compressed_size_bytes_alp;
    sizes[3] = c.compressed_size_bytes_alp_extended;
    flsgpu::host::free_column(c);
    return 0;
  } catch (alp::EncodingException &) {
    return 1;
  }
}
extern "C" int ref_alp_encode_f64(const double *in, size_t n_values, uint64_t *packed, uint8_t *bw,
                       size_t *offs, uint64_t *bases, uint8_t *fac, uint8_t *exp,
                       size_t *exc_offs, double *exc, uint16_t *pos, uint16_t *counts,
                       size_t *sizes) {
  return encode_impl<double, uint64_t>(in, n_values, packed, bw, offs, bases, fac, exp, exc_offs,
                                       exc, pos, counts, sizes);
}
extern "C" int ref_alp_encode_f32(const float *in, size_t n_values, uint32_t *packed, uint8_t *bw,
                       size_t *offs, uint32_t *bases, uint8_t *fac, uint8_t *exp,
                       size_t *exc_offs, float *exc, uint16_t *pos, uint16_t *counts,
                       size_t *sizes) {
  return encode_impl<float, uint32_t>(in, n_values, packed, bw, offs, bases, fac, exp, exc_offs,
                                      exc, pos, counts, sizes);
}

// encoder::init (first-level sample + find_top_k_combinations) on a
// rowgroup; returns k, or -1 when the scheme becomes ALP-RD.
template <typename T>
static int topk_impl(const T *rg, size_t n, uint8_t *ke, uint8_t *kf) {
  std::vector<T> smp(n + 64);
  alp::state<T> st;
  alp::encoder<T>::init(rg, 0, n, smp.data(), st);
  if (st.scheme != alp::Scheme::ALP) return -1;
  for (size_t i = 0; i < st.k_combinations; ++i) {
    ke[i] = (uint8_t)st.best_k_combinations[i].first;
    kf[i] = (uint8_t)st.best_k_combinations[i].second;
  }
  return (int)st.k_combinations;
}
extern "C" int ref_alp_topk_f64(const double *rg, size_t n, uint8_t *ke, uint8_t *kf) { return topk_impl(rg, n, ke, kf); }
extern "C" int ref_alp_topk_f32(const float *rg, size_t n, uint8_t *ke, uint8_t *kf) { return topk_impl(rg, n, ke, kf); }

// encoder::encode for one vector with given top-k candidates (second-level
// choice + encode_simdized).  Returns the exception count.
extern "C" int ref_alp_encode_vector_f64(const double *vec, int k, const uint8_t *ke, const uint8_t *kf,
                              int64_t *encoded, double *exc, uint16_t *pos, uint8_t *out_exp,
                              uint8_t *out_fac) {
  alp::state<double> st;
  st.k_combinations = (uint16_t)k;
  st.best_k_combinations.clear();
  for (int i = 0; i < k; ++i) st.best_k_combinations.emplace_back(ke[i], kf[i]);
  uint16_t count = 0;
  alp::encoder<double>::encode(vec, exc, pos, &count, encoded, st);
  *out_exp = st.exp;
  *out_fac = st.fac;
  return count;
}

// rd_encoder::init / encode / decode, src/alp/rd.hpp.
extern "C" int ref_rd_init_f64(const double *rg, size_t n, uint8_t *rbw, uint8_t *lbw, uint8_t *dsize,
                    uint16_t *dict) {
  std::vector<double> smp(n + 64);
  alp::state<double> st;
  alp::rd_encoder<double>::init(const_cast<double *>(rg), 0, n, smp.data(), st);
  *rbw = st.right_bit_width;
  *lbw = st.left_bit_width;
  *dsize = st.actual_dictionary_size;
  for (int i = 0; i < 8; ++i) dict[i] = st.left_parts_dict[i];
  return 0;
}
// Encode then decode one vector with the dictionary chosen from `rg`.
extern "C" int ref_rd_roundtrip_f64(const double *rg, size_t n, const double *vec, uint64_t *right,
                         uint16_t *left, uint16_t *exc, uint16_t *pos, double *out) {
  std::vector<double> smp(n + 64);
  alp::state<double> st;
  alp::rd_encoder<double>::init(const_cast<double *>(rg), 0, n, smp.data(), st);
  uint16_t count = 0;
  alp::rd_encoder<double>::encode(vec, exc, pos, &count, right, left, st);
  std::vector<uint64_t> r(right, right + 1024);
  std::vector<uint16_t> l(left, left + 1024);
  alp::rd_encoder<double>::decode(out, r.data(), l.data(), exc, pos, &count, st);
  return count;
}

