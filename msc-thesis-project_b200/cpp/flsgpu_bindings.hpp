// flsgpu_bindings.hpp -- the reference's C++ decode API over the C ABI.
//
// Header-only C++17 shim that re-exposes the reference's generated bindings
// (src/generated-bindings/kernel-bindings.cuh:11-175) and column structs
// (src/flsgpu/structs.cuh:33-405) on top of include/flsgpu_b200.h, so code
// written against the reference compiles against this library:
//
//   flsgpu::host::FFORColumn<uint32_t> h = ...;             // host arrays
//   auto d = h.copy_to_device();                            // device column
//   uint32_t *out = bindings::decompress_column<uint32_t>(d, 1, 1,
//                       enums::Unpacker::StatefulBranchless,
//                       enums::Patcher::None, 1);           // new T[n]
//   flsgpu::host::free_column(d); delete[] out;
//
// Semantics follow the reference's host launchers (src/engine/kernels.cuh:
// 94-153): the kernel runs n_samples times with a device synchronisation
// after each, results come back as host arrays the caller deletes.  Errors
// throw std::invalid_argument (argument / binding errors, as the generated
// bindings do, generate-kernel-bindings.py:209) or std::runtime_error (CUDA
// errors, where the reference calls exit(), host-utils.cuh:12-20).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#include "../../include/flsgpu_b200.h"

namespace enums {
// src/engine/enums.cuh:8-53 (same order as the C enums)
enum class DataType { U32, U64, F32, F64 };
enum class Kernel { Decompress, Query, QueryMultiColumn };
enum class Unpacker {
  Dummy, OldFls, SwitchCase, Stateless, StatelessBranchless, StatefulCache, StatefulLocal1,
  StatefulLocal2, StatefulLocal4, StatefulShared1, StatefulShared2, StatefulShared4,
  StatefulRegister1, StatefulRegister2, StatefulRegister4, StatefulRegisterBranchless1,
  StatefulRegisterBranchless2, StatefulRegisterBranchless4, StatefulBranchless,
};
enum class Patcher {
  None, Dummy, Stateless, Stateful, Naive, NaiveBranchless, PrefetchPosition, PrefetchAll,
  PrefetchAllBranchless,
};
}  // namespace enums

using vbw_t = uint8_t;

namespace flsgpu {
namespace detail {
template <typename T> struct same_width_uint {
  using type = typename std::conditional<sizeof(T) == 8, uint64_t, uint32_t>::type;
};
template <typename T> struct same_width_int {
  using type = typename std::conditional<sizeof(T) == 8, int64_t, int32_t>::type;
};
inline void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
inline void check(flsgpu_status s) {
  if (s == FLSGPU_OK) return;
  if (s == FLSGPU_ERR_CUDA || s == FLSGPU_ERR_OUT_OF_MEMORY || s == FLSGPU_ERR_TIMEOUT)
    throw std::runtime_error(flsgpu_last_error());
  throw std::invalid_argument(flsgpu_last_error());
}
template <typename T> T *to_device(const T *host, size_t n, size_t extra = 0) {
  T *d = nullptr;
  cuda_check(cudaMalloc(reinterpret_cast<void **>(&d), (n + extra) * sizeof(T) + 16), "cudaMalloc");
  if (n) cuda_check(cudaMemcpy(d, host, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy");
  return d;
}
template <typename T> void free_device(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}
inline size_t n_vecs_of(size_t n_values) { return (n_values + 1023) / 1024; }
}  // namespace detail

namespace device {
// structs.cuh:33-84, field for field (static_asserts below)
template <typename T> struct BPColumn {
  using UINT_T = typename detail::same_width_uint<T>::type;
  size_t n_values;
  size_t n_vecs;
  UINT_T *packed_array;
  vbw_t *bit_widths;
  size_t *vector_offsets;
};
template <typename T> struct FFORColumn {
  using UINT_T = typename detail::same_width_uint<T>::type;
  size_t n_values;
  BPColumn<T> bp;
  UINT_T *bases;
};
template <typename T> struct ALPColumn {
  using INT_T = typename detail::same_width_int<T>::type;
  using UINT_T = typename detail::same_width_uint<T>::type;
  size_t n_values;
  FFORColumn<UINT_T> ffor;
  INT_T *factors;
  T *fractions;
  uint8_t *factor_indices;
  uint8_t *fraction_indices;
  size_t n_exceptions;
  size_t *exceptions_offsets;
  T *exceptions;
  uint16_t *positions;
  uint16_t *counts;
};
template <typename T> struct ALPExtendedColumn {
  using INT_T = typename detail::same_width_int<T>::type;
  using UINT_T = typename detail::same_width_uint<T>::type;
  size_t n_values;
  FFORColumn<UINT_T> ffor;
  INT_T *factors;
  T *fractions;
  uint8_t *factor_indices;
  uint8_t *fraction_indices;
  size_t n_exceptions;
  size_t *exceptions_offsets;
  T *exceptions;
  uint16_t *positions;
  uint16_t *offsets_counts;
};
static_assert(sizeof(BPColumn<uint32_t>) == sizeof(flsgpu_bp_column), "BPColumn layout");
static_assert(sizeof(FFORColumn<uint64_t>) == sizeof(flsgpu_ffor_column), "FFORColumn layout");
static_assert(sizeof(ALPColumn<double>) == sizeof(flsgpu_alp_column), "ALPColumn layout");
static_assert(sizeof(ALPExtendedColumn<float>) == sizeof(flsgpu_alpx_column), "ALPX layout");
static_assert(offsetof(ALPColumn<double>, counts) == offsetof(flsgpu_alp_column, counts), "");
static_assert(offsetof(ALPExtendedColumn<double>, offsets_counts) ==
                  offsetof(flsgpu_alpx_column, offsets_counts), "");
}  // namespace device

namespace host {
// structs.cuh:89-332: host columns and copy_to_device (with the reference's
// over-read pad after the packed array, structs.cuh:104-105).
template <typename T> struct BPColumn {
  using UINT_T = typename detail::same_width_uint<T>::type;
  using DeviceColumnT = device::BPColumn<T>;
  size_t n_values;
  size_t n_packed_values;
  UINT_T *packed_array;
  vbw_t *bit_widths;
  size_t *vector_offsets;
  size_t get_n_values() const { return n_values; }
  size_t get_n_vecs() const { return detail::n_vecs_of(n_values); }
  device::BPColumn<T> copy_to_device() const {
    const size_t pad = sizeof(T) * (1024 / (8 * sizeof(T))) * 4;
    return device::BPColumn<T>{n_values, get_n_vecs(),
                               detail::to_device(packed_array, n_packed_values, pad),
                               detail::to_device(bit_widths, get_n_vecs()),
                               detail::to_device(vector_offsets, get_n_vecs())};
  }
};
template <typename T> struct FFORColumn {
  using UINT_T = typename detail::same_width_uint<T>::type;
  using DeviceColumnT = device::FFORColumn<T>;
  BPColumn<T> bp;
  UINT_T *bases;
  size_t get_n_values() const { return bp.n_values; }
  size_t get_n_vecs() const { return bp.get_n_vecs(); }
  device::FFORColumn<T> copy_to_device() const {
    return device::FFORColumn<T>{get_n_values(), bp.copy_to_device(),
                                 detail::to_device(bases, get_n_vecs())};
  }
};
template <typename T, bool EXTENDED> struct ALPColumnBase {
  using INT_T = typename detail::same_width_int<T>::type;
  using UINT_T = typename detail::same_width_uint<T>::type;
  FFORColumn<UINT_T> ffor;
  uint8_t *factor_indices;
  uint8_t *fraction_indices;
  size_t n_exceptions;
  size_t *exceptions_offsets;
  T *exceptions;
  uint16_t *positions;
  uint16_t *counts_or_offsets_counts;
  size_t get_n_values() const { return ffor.bp.n_values; }
  size_t get_n_vecs() const { return ffor.bp.get_n_vecs(); }
};
template <typename T> struct ALPExtendedColumn;
template <typename T> struct ALPColumn : ALPColumnBase<T, false> {
  using DeviceColumnT = device::ALPColumn<T>;
  // create_extended_column (structs.cuh:231-308): the same column with its
  // exceptions regrouped by lane, converted on the GPU
  // (flsgpu_alp_to_extended_*).  The result shares ffor and the per-vector
  // metadata with this column; its exceptions, positions and
  // offsets_counts are new malloc'ed host arrays (release with free()).
  ALPExtendedColumn<T> create_extended_column() const;
  device::ALPColumn<T> copy_to_device() const {
    const size_t nv = this->get_n_vecs();
    return device::ALPColumn<T>{this->get_n_values(), this->ffor.copy_to_device(), nullptr,
                                nullptr, detail::to_device(this->factor_indices, nv),
                                detail::to_device(this->fraction_indices, nv), this->n_exceptions,
                                detail::to_device(this->exceptions_offsets, nv),
                                detail::to_device(this->exceptions, this->n_exceptions),
                                detail::to_device(this->positions, this->n_exceptions),
                                detail::to_device(this->counts_or_offsets_counts, nv)};
  }
};
template <typename T> struct ALPExtendedColumn : ALPColumnBase<T, true> {
  using DeviceColumnT = device::ALPExtendedColumn<T>;
  device::ALPExtendedColumn<T> copy_to_device() const {
    const size_t nv = this->get_n_vecs();
    const size_t nl = 1024 / (8 * sizeof(T));
    return device::ALPExtendedColumn<T>{
        this->get_n_values(), this->ffor.copy_to_device(), nullptr, nullptr,
        detail::to_device(this->factor_indices, nv), detail::to_device(this->fraction_indices, nv),
        this->n_exceptions, detail::to_device(this->exceptions_offsets, nv),
        detail::to_device(this->exceptions, this->n_exceptions),
        detail::to_device(this->positions, this->n_exceptions),
        detail::to_device(this->counts_or_offsets_counts, nv * nl)};
  }
};

template <typename T> ALPExtendedColumn<T> ALPColumn<T>::create_extended_column() const {
  const size_t nv = this->get_n_vecs();
  const size_t nl = 1024 / (8 * sizeof(T));
  const size_t ne = this->n_exceptions;
  // the conversion reads only the exception arrays, counts and offsets
  flsgpu_alp_column d{};
  d.n_values = this->get_n_values();
  d.n_exceptions = ne;
  d.exceptions_offsets = detail::to_device(this->exceptions_offsets, nv);
  d.exceptions = detail::to_device(this->exceptions, ne);
  d.positions = detail::to_device(this->positions, ne);
  d.counts = detail::to_device(this->counts_or_offsets_counts, nv);
  T *d_exc = nullptr;
  uint16_t *d_pos = nullptr, *d_oc = nullptr;
  detail::cuda_check(cudaMalloc(reinterpret_cast<void **>(&d_exc), (ne ? ne : 1) * sizeof(T)), "cudaMalloc");
  detail::cuda_check(cudaMalloc(reinterpret_cast<void **>(&d_pos), (ne ? ne : 1) * 2), "cudaMalloc");
  detail::cuda_check(cudaMalloc(reinterpret_cast<void **>(&d_oc), (nv ? nv * nl : 1) * 2), "cudaMalloc");
  flsgpu_alpx_column x{};
  flsgpu_status st;
  if constexpr (sizeof(T) == 8)
    st = flsgpu_alp_to_extended_f64(&d, d_exc, d_pos, d_oc, &x, nullptr);
  else
    st = flsgpu_alp_to_extended_f32(&d, d_exc, d_pos, d_oc, &x, nullptr);
  ALPExtendedColumn<T> out{};
  out.ffor = this->ffor;
  out.factor_indices = this->factor_indices;
  out.fraction_indices = this->fraction_indices;
  out.n_exceptions = ne;
  out.exceptions_offsets = this->exceptions_offsets;
  out.exceptions = static_cast<T *>(malloc(sizeof(T) * (ne ? ne : 1)));
  out.positions = static_cast<uint16_t *>(malloc(2 * (ne ? ne : 1)));
  out.counts_or_offsets_counts = static_cast<uint16_t *>(malloc(2 * (nv ? nv * nl : 1)));
  cudaError_t e = st == FLSGPU_OK ? cudaDeviceSynchronize() : cudaSuccess;
  if (st == FLSGPU_OK && e == cudaSuccess) {
    if (ne) e = cudaMemcpy(out.exceptions, d_exc, sizeof(T) * ne, cudaMemcpyDeviceToHost);
    if (ne && e == cudaSuccess) e = cudaMemcpy(out.positions, d_pos, 2 * ne, cudaMemcpyDeviceToHost);
    if (nv && e == cudaSuccess)
      e = cudaMemcpy(out.counts_or_offsets_counts, d_oc, 2 * nv * nl, cudaMemcpyDeviceToHost);
  }
  for (void *p : {(void *)d.exceptions_offsets, (void *)d.exceptions, (void *)d.positions,
                  (void *)d.counts, (void *)d_exc, (void *)d_pos, (void *)d_oc})
    cudaFree(p);
  detail::check(st);
  detail::cuda_check(e, "create_extended_column");
  return out;
}

// host::free_column(device::...) (structs.cuh:367-400)
template <typename T> void free_column(device::BPColumn<T> c) {
  detail::free_device(c.packed_array);
  detail::free_device(c.bit_widths);
  detail::free_device(c.vector_offsets);
}
template <typename T> void free_column(device::FFORColumn<T> c) {
  free_column(c.bp);
  detail::free_device(c.bases);
}
template <typename C> void free_alp_column(C c) {
  free_column(c.ffor);
  detail::free_device(c.factor_indices);
  detail::free_device(c.fraction_indices);
  detail::free_device(c.exceptions_offsets);
  detail::free_device(c.exceptions);
  detail::free_device(c.positions);
}
template <typename T> void free_column(device::ALPColumn<T> c) {
  free_alp_column(c);
  detail::free_device(c.counts);
}
template <typename T> void free_column(device::ALPExtendedColumn<T> c) {
  free_alp_column(c);
  detail::free_device(c.offsets_counts);
}
}  // namespace host
}  // namespace flsgpu

namespace data {
namespace arrays {
// data::arrays::read_file_as (src/engine/data.cuh:184-232): a binary file of
// T values as a host column of `input_count` values (0: the whole file),
// rounded down to whole vectors of 1024; when the file holds fewer values
// than asked for, its values are repeated until the column is full.  The
// array is new T[count] (release with delete[]).  Throws
// std::invalid_argument when the file cannot be opened or read, when its
// size is not a multiple of sizeof(T), or when it is empty but values are
// asked for (where the reference would loop forever).
template <typename T>
std::pair<T *, size_t> read_file_as(const std::string path, const size_t input_count) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) throw std::invalid_argument("could not open " + path);
  const std::streamsize file_size = f.tellg();
  f.seekg(0, std::ios::beg);
  if ((size_t)file_size % sizeof(T) != 0)
    throw std::invalid_argument("file size is not a multiple of the value size");
  const size_t in_file = (size_t)file_size / sizeof(T);
  size_t count = input_count == 0 ? in_file : input_count;
  count -= count % 1024;
  if (count && !in_file) throw std::invalid_argument("empty file");
  T *column = new T[count ? count : 1];
  const size_t n_read = in_file < count ? in_file : count;
  if (n_read && !f.read(reinterpret_cast<char *>(column), (std::streamsize)(n_read * sizeof(T)))) {
    delete[] column;
    throw std::invalid_argument("failed to read " + path);
  }
  for (size_t filled = n_read; filled < count;) {
    const size_t n = (count - filled) < in_file ? (count - filled) : in_file;
    std::memcpy(column + filled, column, n * sizeof(T));
    filled += n;
  }
  return std::make_pair(column, count);
}
}  // namespace arrays
}  // namespace data

namespace bindings {
namespace detail {
inline flsgpu_decode_opts opts(unsigned nvec, unsigned nval, enums::Unpacker u, enums::Patcher p) {
  return flsgpu_decode_opts{nvec, nval, (uint32_t)u, (uint32_t)p, FLSGPU_VARIANT_AUTO, 0, nullptr, 0};
}
// C entry points per column type
inline flsgpu_status dec(const flsgpu::device::BPColumn<uint32_t> &c, uint32_t *o, const flsgpu_decode_opts *op) { return flsgpu_decompress_bp_u32(reinterpret_cast<const flsgpu_bp_column *>(&c), o, op, nullptr); }
inline flsgpu_status dec(const flsgpu::device::BPColumn<uint64_t> &c, uint64_t *o, const flsgpu_decode_opts *op) { return flsgpu_decompress_bp_u64(reinterpret_cast<const flsgpu_bp_column *>(&c), o, op, nullptr); }
inline flsgpu_status dec(const flsgpu::device::FFORColumn<uint32_t> &c, uint32_t *o, const flsgpu_decode_opts *op) { return flsgpu_decompress_ffor_u32(reinterpret_cast<const flsgpu_ffor_column *>(&c), o, op, nullptr); }
inline flsgpu_status dec(const flsgpu::device::FFORColumn<uint64_t> &c, uint64_t *o, const flsgpu_decode_opts *op) { return flsgpu_decompress_ffor_u64(reinterpret_cast<const flsgpu_ffor_column *>(&c), o, op, nullptr); }
inline flsgpu_status dec(const flsgpu::device::ALPColumn<float> &c, float *o, const flsgpu_decode_opts *op) { return flsgpu_decompress_alp_f32(reinterpret_cast<const flsgpu_alp_column *>(&c), o, op, nullptr); }
inline flsgpu_status dec(const flsgpu::device::ALPColumn<double> &c, double *o, const flsgpu_decode_opts *op) { return flsgpu_decompress_alp_f64(reinterpret_cast<const flsgpu_alp_column *>(&c), o, op, nullptr); }
inline flsgpu_status dec(const flsgpu::device::ALPExtendedColumn<float> &c, float *o, const flsgpu_decode_opts *op) { return flsgpu_decompress_alpx_f32(reinterpret_cast<const flsgpu_alpx_column *>(&c), o, op, nullptr); }
inline flsgpu_status dec(const flsgpu::device::ALPExtendedColumn<double> &c, double *o, const flsgpu_decode_opts *op) { return flsgpu_decompress_alpx_f64(reinterpret_cast<const flsgpu_alpx_column *>(&c), o, op, nullptr); }
inline flsgpu_status qry(const flsgpu::device::BPColumn<uint32_t> &c, uint32_t m, uint8_t *f, const flsgpu_decode_opts *op) { return flsgpu_query_bp_u32(reinterpret_cast<const flsgpu_bp_column *>(&c), m, f, op, nullptr); }
inline flsgpu_status qry(const flsgpu::device::BPColumn<uint64_t> &c, uint64_t m, uint8_t *f, const flsgpu_decode_opts *op) { return flsgpu_query_bp_u64(reinterpret_cast<const flsgpu_bp_column *>(&c), m, f, op, nullptr); }
inline flsgpu_status qry(const flsgpu::device::FFORColumn<uint32_t> &c, uint32_t m, uint8_t *f, const flsgpu_decode_opts *op) { return flsgpu_query_ffor_u32(reinterpret_cast<const flsgpu_ffor_column *>(&c), m, f, op, nullptr); }
inline flsgpu_status qry(const flsgpu::device::FFORColumn<uint64_t> &c, uint64_t m, uint8_t *f, const flsgpu_decode_opts *op) { return flsgpu_query_ffor_u64(reinterpret_cast<const flsgpu_ffor_column *>(&c), m, f, op, nullptr); }
inline flsgpu_status qry(const flsgpu::device::ALPColumn<float> &c, float m, uint8_t *f, const flsgpu_decode_opts *op) { return flsgpu_query_alp_f32(reinterpret_cast<const flsgpu_alp_column *>(&c), m, f, op, nullptr); }
inline flsgpu_status qry(const flsgpu::device::ALPColumn<double> &c, double m, uint8_t *f, const flsgpu_decode_opts *op) { return flsgpu_query_alp_f64(reinterpret_cast<const flsgpu_alp_column *>(&c), m, f, op, nullptr); }
inline flsgpu_status qry(const flsgpu::device::ALPExtendedColumn<float> &c, float m, uint8_t *f, const flsgpu_decode_opts *op) { return flsgpu_query_alpx_f32(reinterpret_cast<const flsgpu_alpx_column *>(&c), m, f, op, nullptr); }
inline flsgpu_status qry(const flsgpu::device::ALPExtendedColumn<double> &c, double m, uint8_t *f, const flsgpu_decode_opts *op) { return flsgpu_query_alpx_f64(reinterpret_cast<const flsgpu_alpx_column *>(&c), m, f, op, nullptr); }
template <typename T> struct DeviceBuf {
  T *p = nullptr;
  explicit DeviceBuf(size_t n) { flsgpu::detail::cuda_check(cudaMalloc(reinterpret_cast<void **>(&p), n * sizeof(T) + 16), "cudaMalloc"); }
  ~DeviceBuf() { if (p) cudaFree(p); }
};
}  // namespace detail

// bindings::decompress_column (kernel-bindings.cuh:11-15, :42-90)
template <typename T, typename ColumnT>
T *decompress_column(const ColumnT column, const unsigned unpack_n_vectors,
                     const unsigned unpack_n_values, const enums::Unpacker unpacker,
                     const enums::Patcher patcher, const uint32_t n_samples) {
  const auto o = detail::opts(unpack_n_vectors, unpack_n_values, unpacker, patcher);
  detail::DeviceBuf<T> d(column.n_values);
  for (uint32_t i = 0; i < n_samples; ++i) {
    flsgpu::detail::check(detail::dec(column, d.p, &o));
    flsgpu::detail::cuda_check(cudaDeviceSynchronize(), "decompress_column");
  }
  T *out = new T[column.n_values];
  flsgpu::detail::cuda_check(cudaMemcpy(out, d.p, sizeof(T) * column.n_values, cudaMemcpyDeviceToHost), "copy");
  return out;
}

// bindings::query_column (kernel-bindings.cuh:17-21, :92-131)
template <typename T, typename ColumnT>
bool query_column(const ColumnT column, const unsigned unpack_n_vectors,
                  const unsigned unpack_n_values, const enums::Unpacker unpacker,
                  const enums::Patcher patcher, const T magic_value, const uint32_t n_samples) {
  const auto o = detail::opts(unpack_n_vectors, unpack_n_values, unpacker, patcher);
  detail::DeviceBuf<uint8_t> d(1);
  flsgpu::detail::cuda_check(cudaMemset(d.p, 0, 1), "memset");
  for (uint32_t i = 0; i < n_samples; ++i) {
    flsgpu::detail::check(detail::qry(column, magic_value, d.p, &o));
    flsgpu::detail::cuda_check(cudaDeviceSynchronize(), "query_column");
  }
  uint8_t h = 0;
  flsgpu::detail::cuda_check(cudaMemcpy(&h, d.p, 1, cudaMemcpyDeviceToHost), "copy");
  return h != 0;
}

namespace detail {
inline flsgpu_status qmc(const flsgpu::device::FFORColumn<uint32_t> *c, uint32_t n, uint32_t v, uint8_t *o, const flsgpu_decode_opts *op) { return flsgpu_query_multi_column_ffor_u32(reinterpret_cast<const flsgpu_ffor_column *>(c), n, v, o, op, nullptr); }
inline flsgpu_status qmc(const flsgpu::device::FFORColumn<uint64_t> *c, uint32_t n, uint64_t v, uint8_t *o, const flsgpu_decode_opts *op) { return flsgpu_query_multi_column_ffor_u64(reinterpret_cast<const flsgpu_ffor_column *>(c), n, v, o, op, nullptr); }
inline flsgpu_status qmc(const flsgpu::device::ALPColumn<float> *c, uint32_t n, float v, uint8_t *o, const flsgpu_decode_opts *op) { return flsgpu_query_multi_column_alp_f32(reinterpret_cast<const flsgpu_alp_column *>(c), n, v, o, op, nullptr); }
inline flsgpu_status qmc(const flsgpu::device::ALPColumn<double> *c, uint32_t n, double v, uint8_t *o, const flsgpu_decode_opts *op) { return flsgpu_query_multi_column_alp_f64(reinterpret_cast<const flsgpu_alp_column *>(c), n, v, o, op, nullptr); }
template <typename C> auto &bp_of(C &c) { return c.bp; }
template <typename T> auto &bp_of(flsgpu::host::ALPColumn<T> &c) { return c.ffor.bp; }
}  // namespace detail

// bindings::query_multi_column (kernel-bindings.cuh:30-35) and its host
// harness kernels::host::query_multi_column (src/engine/multi-column-host-
// kernels.cuh:13-123): ten device copies of the host column, each after the
// bit widths were shuffled (data.cuh:521-531: a random permutation of the
// widths, vector offsets recomputed as their prefix sum, so every copy is a
// column of the same packed size), then the multi-column scan over the
// first 1, 2, ..., 10 copies, n_samples times each with a device
// synchronisation after every launch; the result is set when any of those
// scans found a lane equal to magic_value in every column.  The shuffle
// works on a copy of the widths (the reference permutes the caller's array
// in place and keeps the old offsets).  Host column types: FFORColumn<u32 /
// u64>, ALPColumn<float / double>.
template <typename T, typename HostColumnT>
bool query_multi_column(HostColumnT column, const unsigned unpack_n_vectors,
                        const unsigned unpack_n_values, const enums::Unpacker unpacker,
                        const enums::Patcher patcher, const T magic_value,
                        const uint32_t n_samples) {
  using DeviceColumnT = typename HostColumnT::DeviceColumnT;
  constexpr int MAX_N_COLS = 10;
  auto &bp = detail::bp_of(column);
  const size_t nv = bp.get_n_vecs();
  using UINT_T = typename flsgpu::detail::same_width_uint<T>::type;
  constexpr size_t NL = 1024 / (8 * sizeof(UINT_T));
  vbw_t *orig_bw = bp.bit_widths;
  size_t *orig_offs = bp.vector_offsets;
  vbw_t *bw = new vbw_t[nv ? nv : 1];
  size_t *offs = new size_t[nv ? nv : 1];
  std::memcpy(bw, orig_bw, nv);
  std::random_device rd;
  std::default_random_engine rng(rd());
  DeviceColumnT dev[MAX_N_COLS];
  for (int c = 0; c < MAX_N_COLS; ++c) {
    std::shuffle(bw, bw + nv, rng);
    size_t acc = 0;
    for (size_t v = 0; v < nv; ++v) {
      offs[v] = acc;
      acc += (size_t)bw[v] * NL;
    }
    bp.bit_widths = bw;
    bp.vector_offsets = offs;
    dev[c] = column.copy_to_device();
  }
  bp.bit_widths = orig_bw;
  bp.vector_offsets = orig_offs;
  delete[] bw;
  delete[] offs;
  const auto o = detail::opts(unpack_n_vectors, unpack_n_values, unpacker, patcher);
  detail::DeviceBuf<uint8_t> d(1);
  flsgpu::detail::cuda_check(cudaMemset(d.p, 0, 1), "memset");
  for (uint32_t n = 1; n <= (uint32_t)MAX_N_COLS; ++n)
    for (uint32_t i = 0; i < n_samples; ++i) {
      flsgpu::detail::check(detail::qmc(dev, n, magic_value, d.p, &o));
      flsgpu::detail::cuda_check(cudaDeviceSynchronize(), "query_multi_column");
    }
  for (int c = 0; c < MAX_N_COLS; ++c) flsgpu::host::free_column(dev[c]);
  uint8_t h = 0;
  flsgpu::detail::cuda_check(cudaMemcpy(&h, d.p, 1, cudaMemcpyDeviceToHost), "copy");
  return h != 0;
}

// bindings::compute_column (kernel-bindings.cuh:23-28, :133-144)
template <typename T, typename ColumnT>
bool compute_column(const ColumnT column, const unsigned unpack_n_vectors,
                    const unsigned unpack_n_values, const enums::Unpacker unpacker,
                    const enums::Patcher patcher, const unsigned n_repetitions,
                    const uint32_t n_samples) {
  const auto o = detail::opts(unpack_n_vectors, unpack_n_values, unpacker, patcher);
  detail::DeviceBuf<uint8_t> d(1);
  flsgpu::detail::cuda_check(cudaMemset(d.p, 0, 1), "memset");
  for (uint32_t i = 0; i < n_samples; ++i) {
    flsgpu_status s;
    if constexpr (sizeof(T) == 4)
      s = flsgpu_compute_ffor_u32(reinterpret_cast<const flsgpu_ffor_column *>(&column), n_repetitions, d.p, &o, nullptr);
    else
      s = flsgpu_compute_ffor_u64(reinterpret_cast<const flsgpu_ffor_column *>(&column), n_repetitions, d.p, &o, nullptr);
    flsgpu::detail::check(s);
    flsgpu::detail::cuda_check(cudaDeviceSynchronize(), "compute_column");
  }
  uint8_t h = 0;
  flsgpu::detail::cuda_check(cudaMemcpy(&h, d.p, 1, cudaMemcpyDeviceToHost), "copy");
  return h != 0;
}
}  // namespace bindings
