// compmatmul_b200.hpp -- C++ header entry points with the shapes of the
// reference's header API (matmul_fft.hpp, matmul_fwht.hpp, matmul_sketch.hpp,
// hashing.hpp), forwarding to the C ABI of libcmm_b200.so.  A caller of
//   compmatmul::matmul_fft<compmatmul::multiply_add_shift_hash>(...)
// switches by including this header and using namespace compmatmul_b200.
//
//   reference                                  here
//   matmul_fft<H>(n_a,n_inner,n_b,C,AT,B,d,b,seed)      matmul_fft.hpp:155-178
//   matmul_fwht<H>(...)                                  matmul_fwht.hpp:144-167
//   matmul_compressed_product_fft<H>(n_a,..,seed)->sketch matmul_fft.hpp:25-129
//   matmul_compressed_product_fwht<H>(...)->sketch        matmul_fwht.hpp:25-114
//   matmul_decompress_fft<H>(cols,C,i,j,sketch,scratch)   matmul_fft.hpp:135-147
//   matmul_decompress_fwht<H>(...)                        matmul_fwht.hpp:122-134
//   array::matmul_gemm<double>(n_a,n_inner,n_b,C,AT,B)    array.hpp:85-95
//
// Failures throw the reference's exception types: std::invalid_argument,
// std::runtime_error, std::bad_alloc.  Pointers are host pointers.
#pragma once

#include <cstdint>
#include <new>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "compmatmul_b200.h"

namespace compmatmul_b200 {

// Hash family tags (hashing.hpp:27, 111, 232); the functions themselves are
// drawn inside the library, bit-exact with the reference's draw().
struct multiply_shift_hash { static constexpr int kind = CMM_HASH_MULTIPLY_SHIFT; };
struct multiply_add_shift_hash { static constexpr int kind = CMM_HASH_MULTIPLY_ADD_SHIFT; };
template <int CharBits, typename Key, typename Hash>
struct tabulation_hash {
  static_assert(CharBits == 8 || CharBits == 16, "tabulation over 8- or 16-bit characters");
  static constexpr int kind = CharBits == 8 ? CMM_HASH_TABULATION8 : CMM_HASH_TABULATION16;
};

inline void throw_status(int st) {
  if (st == CMM_OK) return;
  const std::string msg = cmm_last_error();
  if (st == CMM_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
  if (st == CMM_ERR_NO_MEMORY) throw std::bad_alloc();
  throw std::runtime_error(msg);
}

// The compressed product of one call (matmul_sketch.hpp:9-81): d, b, the
// seed the hash functions were drawn with, and p (d x b, row-major).
template <typename Hash>
struct matmul_sketch {
  int d = 0;
  int b = 0;
  uint64_t seed = 0;
  uint32_t mod_mask = 0;
  std::vector<double> p;
};

template <typename Hash>
using matmul_fft_sketch = matmul_sketch<Hash>;
template <typename Hash>
using matmul_fwht_sketch = matmul_sketch<Hash>;

namespace detail {
template <typename Hash>
matmul_sketch<Hash> compressed(int variant, int64_t n_a, int64_t n_inner, int64_t n_b,
                               const double* A, const double* B, int d, int b,
                               std::optional<uint64_t> seed) {
  matmul_sketch<Hash> s;
  s.d = d;
  s.b = b;
  s.mod_mask = (uint32_t)b - 1u;
  s.p.assign((size_t)(d > 0 ? d : 0) * (size_t)(b > 0 ? b : 0), 0.0);
  uint64_t used = 0;
  throw_status(cmm_compressed_product(variant, Hash::kind, n_a, n_inner, n_b, A, B, d, b,
                                      seed ? 1 : 0, seed.value_or(0), s.p.data(), &used));
  s.seed = used;
  return s;
}

template <typename Hash>
void decompress(int variant, int cols, double* C, uint32_t i, uint32_t j,
                const matmul_sketch<Hash>& sk, double* /*scratch*/) {
  double out = 0.0;
  throw_status(cmm_decompress(variant, Hash::kind, sk.d, sk.b, sk.seed, sk.p.data(), 1, &i, &j, &out));
  C[(size_t)i * (size_t)cols + j] = out;
}
}  // namespace detail

template <typename Hash>
matmul_fft_sketch<Hash> matmul_compressed_product_fft(int n_a, int n_inner, int n_b,
                                                      const double* A, const double* B, int d,
                                                      int b, std::optional<uint64_t> seed = std::nullopt) {
  return detail::compressed<Hash>(CMM_VARIANT_FFT, n_a, n_inner, n_b, A, B, d, b, seed);
}

template <typename Hash>
matmul_fwht_sketch<Hash> matmul_compressed_product_fwht(int n_a, int n_inner, int n_b,
                                                        const double* A, const double* B, int d,
                                                        int b, std::optional<uint64_t> seed = std::nullopt) {
  return detail::compressed<Hash>(CMM_VARIANT_FWHT, n_a, n_inner, n_b, A, B, d, b, seed);
}

// One entry per call, like the reference; prefer decompress_entries for many.
template <typename Hash>
void matmul_decompress_fft(int cols, double* C, uint32_t i, uint32_t j,
                           const matmul_fft_sketch<Hash>& sketch, double* scratch) {
  detail::decompress<Hash>(CMM_VARIANT_FFT, cols, C, i, j, sketch, scratch);
}

template <typename Hash>
void matmul_decompress_fwht(int cols, double* C, uint32_t i, uint32_t j,
                            const matmul_fwht_sketch<Hash>& sketch, double* scratch) {
  detail::decompress<Hash>(CMM_VARIANT_FWHT, cols, C, i, j, sketch, scratch);
}

// Batched form: out[e] = estimate of C[i[e]][j[e]] (one device launch).
template <typename Hash>
void decompress_entries(int variant, const matmul_sketch<Hash>& sketch, int64_t count,
                        const uint32_t* i, const uint32_t* j, double* out) {
  throw_status(cmm_decompress(variant, Hash::kind, sketch.d, sketch.b, sketch.seed,
                              sketch.p.data(), count, i, j, out));
}

template <typename Hash>
void matmul_fft(int n_a, int n_inner, int n_b, double* C, const double* AT, const double* B, int d,
                int b, std::optional<uint64_t> seed = std::nullopt) {
  throw_status(cmm_matmul(CMM_VARIANT_FFT, Hash::kind, n_a, n_inner, n_b, C, AT, B, d, b,
                          seed ? 1 : 0, seed.value_or(0)));
}

template <typename Hash>
void matmul_fwht(int n_a, int n_inner, int n_b, double* C, const double* AT, const double* B,
                 int d, int b, std::optional<uint64_t> seed = std::nullopt) {
  throw_status(cmm_matmul(CMM_VARIANT_FWHT, Hash::kind, n_a, n_inner, n_b, C, AT, B, d, b,
                          seed ? 1 : 0, seed.value_or(0)));
}

namespace array {
template <typename T>
void matmul_gemm(int n_a, int n_inner, int n_b, T* C, const T* AT, const T* B);
template <>
inline void matmul_gemm<double>(int n_a, int n_inner, int n_b, double* C, const double* AT,
                                const double* B) {
  throw_status(cmm_gemm(n_a, n_inner, n_b, C, AT, B));
}
}  // namespace array

}  // namespace compmatmul_b200
