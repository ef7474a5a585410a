// shim_consumer.cu -- test program for the C++ drop-in shim
// (msc-thesis-project_b200/cpp/flsgpu_bindings.hpp): code written against
// the reference's API (host columns, copy_to_device, bindings::*,
// host::free_column), exported as C functions for the parity tests.  Each
// returns 0, or 1 when the shim threw (the message goes to stderr).
#include <cstdio>
#include <exception>

#include "../../msc-thesis-project_b200/cpp/flsgpu_bindings.hpp"

template <typename F> static int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "shim: %s\n", e.what());
    return 1;
  }
}

template <typename T>
static flsgpu::host::FFORColumn<T> host_ffor(const T *packed, size_t n_packed, const uint8_t *bw,
                                             const size_t *offs, const T *bases, size_t n_values) {
  flsgpu::host::FFORColumn<T> h{};
  h.bp.n_values = n_values;
  h.bp.n_packed_values = n_packed;
  h.bp.packed_array = const_cast<T *>(packed);
  h.bp.bit_widths = const_cast<uint8_t *>(bw);
  h.bp.vector_offsets = const_cast<size_t *>(offs);
  h.bases = const_cast<T *>(bases);
  return h;
}

template <typename T>
static flsgpu::host::ALPColumn<T> host_alp(
    const typename flsgpu::detail::same_width_uint<T>::type *packed, size_t n_packed,
    const uint8_t *bw, const size_t *offs, const typename flsgpu::detail::same_width_uint<T>::type *bases,
    size_t n_values, const uint8_t *fac, const uint8_t *frac, size_t n_exc, const size_t *eoffs,
    const T *exc, const uint16_t *pos, const uint16_t *counts) {
  using U = typename flsgpu::detail::same_width_uint<T>::type;
  flsgpu::host::ALPColumn<T> h{};
  h.ffor = host_ffor<U>(packed, n_packed, bw, offs, bases, n_values);
  h.factor_indices = const_cast<uint8_t *>(fac);
  h.fraction_indices = const_cast<uint8_t *>(frac);
  h.n_exceptions = n_exc;
  h.exceptions_offsets = const_cast<size_t *>(eoffs);
  h.exceptions = const_cast<T *>(exc);
  h.positions = const_cast<uint16_t *>(pos);
  h.counts_or_offsets_counts = const_cast<uint16_t *>(counts);
  return h;
}

extern "C" {

#define FFOR_DECODE(SUF, T)                                                                  \
  int shim_decompress_ffor_##SUF(const T *packed, size_t n_packed, const uint8_t *bw,      \
                                 const size_t *offs, const T *bases, size_t n_values,       \
                                 T *out) {                                                  \
    return guarded([&] {                                                                    \
      auto d = host_ffor<T>(packed, n_packed, bw, offs, bases, n_values).copy_to_device();  \
      T *r = bindings::decompress_column<T>(d, 1, 1, enums::Unpacker::StatefulBranchless,   \
                                            enums::Patcher::None, 2);                       \
      std::memcpy(out, r, sizeof(T) * n_values);                                            \
      delete[] r;                                                                           \
      flsgpu::host::free_column(d);                                                         \
    });                                                                                     \
  }                                                                                         \
  int shim_query_ffor_##SUF(const T *packed, size_t n_packed, const uint8_t *bw,           \
                            const size_t *offs, const T *bases, size_t n_values, T magic,  \
                            int *found) {                                                   \
    return guarded([&] {                                                                    \
      auto d = host_ffor<T>(packed, n_packed, bw, offs, bases, n_values).copy_to_device();  \
      *found = bindings::query_column<T>(d, 1, 1, enums::Unpacker::StatefulBranchless,      \
                                         enums::Patcher::None, magic, 1);                   \
      flsgpu::host::free_column(d);                                                         \
    });                                                                                     \
  }                                                                                         \
  int shim_compute_ffor_##SUF(const T *packed, size_t n_packed, const uint8_t *bw,         \
                              const size_t *offs, const T *bases, size_t n_values,          \
                              int *found) {                                                 \
    return guarded([&] {                                                                    \
      auto d = host_ffor<T>(packed, n_packed, bw, offs, bases, n_values).copy_to_device();  \
      *found = bindings::compute_column<T>(d, 1, 1, enums::Unpacker::StatefulBranchless,    \
                                           enums::Patcher::None, 10, 1);                    \
      flsgpu::host::free_column(d);                                                         \
    });                                                                                     \
  }                                                                                         \
  int shim_query_multi_column_ffor_##SUF(const T *packed, size_t n_packed, const uint8_t *bw, \
                                         const size_t *offs, const T *bases, size_t n_values, \
                                         T magic, int *found) {                             \
    return guarded([&] {                                                                    \
      auto h = host_ffor<T>(packed, n_packed, bw, offs, bases, n_values);                   \
      *found = bindings::query_multi_column<T>(h, 1, 1, enums::Unpacker::StatefulBranchless, \
                                               enums::Patcher::None, magic, 1);             \
    });                                                                                     \
  }
FFOR_DECODE(u32, uint32_t)
FFOR_DECODE(u64, uint64_t)

int shim_read_file_f64(const char *path, size_t input_count, double *out, size_t *count) {
  return guarded([&] {
    auto r = data::arrays::read_file_as<double>(path, input_count);
    std::memcpy(out, r.first, sizeof(double) * r.second);
    *count = r.second;
    delete[] r.first;
  });
}

#define ALP_DECODE(SUF, T, U)                                                                 \
  int shim_decompress_alp_##SUF(const U *packed, size_t n_packed, const uint8_t *bw,         \
                                const size_t *offs, const U *bases, size_t n_values,         \
                                const uint8_t *fac, const uint8_t *frac, size_t n_exc,       \
                                const size_t *eoffs, const T *exc, const uint16_t *pos,      \
                                const uint16_t *counts, int extended, T *out) {              \
    return guarded([&] {                                                                     \
      auto h = host_alp<T>(packed, n_packed, bw, offs, bases, n_values, fac, frac, n_exc,    \
                           eoffs, exc, pos, counts);                                         \
      T *r = nullptr;                                                                        \
      if (extended) {                                                                        \
        auto x = h.create_extended_column();                                                 \
        auto d = x.copy_to_device();                                                         \
        r = bindings::decompress_column<T>(d, 1, 1, enums::Unpacker::StatefulBranchless,     \
                                           enums::Patcher::PrefetchAll, 1);                  \
        flsgpu::host::free_column(d);                                                        \
        std::free(x.exceptions);                                                             \
        std::free(x.positions);                                                              \
        std::free(x.counts_or_offsets_counts);                                               \
      } else {                                                                               \
        auto d = h.copy_to_device();                                                         \
        r = bindings::decompress_column<T>(d, 1, 1, enums::Unpacker::StatefulBranchless,     \
                                           enums::Patcher::PrefetchAll, 1);                  \
        flsgpu::host::free_column(d);                                                        \
      }                                                                                      \
      std::memcpy(out, r, sizeof(T) * n_values);                                             \
      delete[] r;                                                                            \
    });                                                                                      \
  }
ALP_DECODE(f32, float, uint32_t)
ALP_DECODE(f64, double, uint64_t)

}  // extern "C"
