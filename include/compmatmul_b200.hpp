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
//   matmul_sketch<H>(d,b,seed), .h1/.h2/.s1/.s2, .p.get() matmul_sketch.hpp:9-81
//   multiply_shift_hash, multiply_add_shift_hash,         hashing.hpp:27-183
//   sign_hash<H>, tabulation_hash<8|16,u32,u32>           hashing.hpp:192-320
//   rng                                                   rng.hpp:51-76
//
// Failures throw the reference's exception types: std::invalid_argument,
// std::runtime_error, std::bad_alloc.  Pointers are host pointers.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <optional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "compmatmul_b200.h"

namespace compmatmul_b200 {

inline void throw_status(int st) {
  if (st == CMM_OK) return;
  const std::string msg = cmm_last_error();
  if (st == CMM_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
  if (st == CMM_ERR_NO_MEMORY) throw std::bad_alloc();
  throw std::runtime_error(msg);
}

namespace detail {
inline bool is_pow2(uint64_t x) { return x > 0 && (x & (x - 1)) == 0; }
inline int ilog2(uint64_t x) {
  int l = -1;
  while (x) {
    x >>= 1;
    ++l;
  }
  return l;
}
inline void check_buckets(size_t buckets) {
  if (!is_pow2(buckets)) throw std::invalid_argument("The number of buckets must be a power of 2");
}
// packed parameters of n functions of one family (cmm_hash_params)
inline std::vector<uint64_t> draw_params(int kind, size_t n, size_t buckets, std::optional<uint64_t> seed,
                                         size_t words_per_fn) {
  check_buckets(buckets);
  std::vector<uint64_t> w(n * words_per_fn + 1);
  throw_status(cmm_hash_params(kind, (int)n, buckets, seed.value_or(cmm_time_millis()), w.data(),
                               w.size() * sizeof(uint64_t)));
  return w;
}
}  // namespace detail

// rng (rng.hpp:51-76): xoshiro256** seeded by splitmix64; without a seed,
// the millisecond clock.
class rng {
 public:
  explicit rng(std::optional<uint64_t> seed = std::nullopt) {
    cmm_rng_seed(seed.value_or(cmm_time_millis()), s_);
  }
  uint64_t operator()() { return cmm_rng_next(s_); }

 private:
  uint64_t s_[4];
};

// The reference's hash families (hashing.hpp), evaluated on the host for
// callers that inspect a sketch's functions; the sketch kernels evaluate
// the same functions on the device.  draw()/draw_one() give the
// reference's parameters bit for bit (same seed, same draw order).

// multiply-shift, hashing.hpp:27-102: h(x) = (a x) >> (64 - log2 buckets),
// sign = top bit of a x
class multiply_shift_hash {
 public:
  using key_t = uint32_t;
  using hash_t = uint32_t;
  using sign_t = int;
  static constexpr int kind = CMM_HASH_MULTIPLY_SHIFT;

  multiply_shift_hash() = default;
  explicit multiply_shift_hash(size_t buckets, uint64_t a)
      : a_(a), shift_(detail::is_pow2(buckets) ? 64 - detail::ilog2(buckets)
                                               : throw std::invalid_argument(
                                                     "The number of buckets must be a power of 2")) {}
  static multiply_shift_hash draw_one(size_t buckets, std::optional<uint64_t> seed = std::nullopt) {
    return draw(1, buckets, seed)[0];
  }
  static std::vector<multiply_shift_hash> draw(size_t n, size_t buckets,
                                               std::optional<uint64_t> seed = std::nullopt) {
    const std::vector<uint64_t> w = detail::draw_params(kind, n, buckets, seed, 1);
    std::vector<multiply_shift_hash> h(n);
    for (size_t f = 0; f < n; ++f) h[f] = multiply_shift_hash(buckets, w[f]);
    return h;
  }
  hash_t operator()(key_t key) const { return (hash_t)((a_ * key) >> shift_); }
  sign_t sign(key_t key) const { return ((a_ * key) >> 63) ? 1 : -1; }
  uint64_t get_a() const { return a_; }

 private:
  uint64_t a_ = 0;
  int shift_ = 64;
};

// multiply-add-shift (the default), hashing.hpp:111-183:
// h(x) = (a x + b) >> (64 - log2 buckets), sign = top bit of a x + b
class multiply_add_shift_hash {
 public:
  using key_t = uint32_t;
  using hash_t = uint32_t;
  using sign_t = int;
  static constexpr int kind = CMM_HASH_MULTIPLY_ADD_SHIFT;

  multiply_add_shift_hash() = default;
  explicit multiply_add_shift_hash(size_t buckets, uint64_t a, uint64_t b)
      : a_(a), b_(b), shift_(detail::is_pow2(buckets) ? 64 - detail::ilog2(buckets)
                                                      : throw std::invalid_argument(
                                                            "The number of buckets must be a power of 2")) {}
  static multiply_add_shift_hash draw_one(size_t buckets, std::optional<uint64_t> seed = std::nullopt) {
    return draw(1, buckets, seed)[0];
  }
  static std::vector<multiply_add_shift_hash> draw(size_t n, size_t buckets,
                                                   std::optional<uint64_t> seed = std::nullopt) {
    const std::vector<uint64_t> w = detail::draw_params(kind, n, buckets, seed, 2);
    std::vector<multiply_add_shift_hash> h(n);
    for (size_t f = 0; f < n; ++f) h[f] = multiply_add_shift_hash(buckets, w[2 * f], w[2 * f + 1]);
    return h;
  }
  hash_t operator()(key_t key) const { return (hash_t)((a_ * key + b_) >> shift_); }
  sign_t sign(key_t key) const { return ((a_ * key + b_) >> 63) ? 1 : -1; }
  uint64_t get_a() const { return a_; }
  uint64_t get_b() const { return b_; }

 private:
  uint64_t a_ = 0, b_ = 0;
  int shift_ = 64;
};

// sign_hash<H>, hashing.hpp:192-228: a function of H with two buckets used
// as a sign, +1 when it hashes to bucket 1
template <typename Hash>
class sign_hash {
 public:
  using key_t = typename Hash::key_t;
  using hash_t = int;
  sign_hash() = default;
  static sign_hash draw_one(std::optional<uint64_t> seed = std::nullopt) {
    return sign_hash(Hash::draw_one(2, seed));
  }
  static std::vector<sign_hash> draw(size_t n, std::optional<uint64_t> seed = std::nullopt) {
    const std::vector<Hash> h = Hash::draw(n, 2, seed);
    std::vector<sign_hash> s;
    s.reserve(n);
    for (const Hash& x : h) s.push_back(sign_hash(x));
    return s;
  }
  hash_t operator()(key_t key) const { return hash_(key) > 0 ? 1 : -1; }

 private:
  explicit sign_hash(const Hash& h) : hash_(h) {}
  Hash hash_;
};

// simple tabulation, hashing.hpp:232-320: XOR of T[c][character c of x],
// >> (bits of Hash - log2 buckets); sign = top bit of the XOR.  The library
// (and the reference's Python binding, compmatmul.cpp:97-104) uses 32-bit
// keys and hash values over 8- or 16-bit characters.
template <int CharBits, typename Key, typename Hash>
class tabulation_hash {
  static_assert(CharBits == 8 || CharBits == 16, "tabulation over 8- or 16-bit characters");
  static_assert(std::is_same<Key, uint32_t>::value && std::is_same<Hash, uint32_t>::value,
                "32-bit keys and hash values");
  static constexpr int kChars = 32 / CharBits;
  static constexpr uint32_t kMask = (uint32_t)((1u << CharBits) - 1u);

 public:
  using key_t = Key;
  using hash_t = Hash;
  using sign_t = int;
  static constexpr int kind = CharBits == 8 ? CMM_HASH_TABULATION8 : CMM_HASH_TABULATION16;

  tabulation_hash() = default;
  tabulation_hash(size_t buckets, const Hash* S)
      : T_(S, S + kChars * (1u << CharBits)),
        shift_(detail::is_pow2(buckets) ? 32 - detail::ilog2(buckets)
                                        : throw std::invalid_argument(
                                              "The number of buckets must be a power of 2")) {}
  static tabulation_hash draw_one(size_t buckets, std::optional<uint64_t> seed = std::nullopt) {
    return draw(1, buckets, seed)[0];
  }
  static std::vector<tabulation_hash> draw(size_t n, size_t buckets, std::optional<uint64_t> seed = std::nullopt) {
    const size_t words = (size_t)kChars * (1u << CharBits);  // u32 table words per function
    const std::vector<uint64_t> w = detail::draw_params(kind, n, buckets, seed, words / 2);
    const Hash* T = reinterpret_cast<const Hash*>(w.data());
    std::vector<tabulation_hash> h;
    h.reserve(n);
    for (size_t f = 0; f < n; ++f) h.emplace_back(buckets, T + f * words);
    return h;
  }
  hash_t operator()(Key key) const { return mix(key) >> shift_; }
  sign_t sign(Key key) const { return (mix(key) >> 31) ? 1 : -1; }

 private:
  uint32_t mix(uint32_t key) const {
    uint32_t h = 0;
    for (int c = 0; c < kChars; ++c) h ^= T_[(size_t)c * (1u << CharBits) + ((key >> (c * CharBits)) & kMask)];
    return h;
  }
  std::vector<Hash> T_;  // T[c][v], row-major
  int shift_ = 32;
};

// matmul_sketch<H>, matmul_sketch.hpp:9-81: d repetitions over b buckets,
// the hash functions h1 <- seed, h2 <- seed + 1, s1 <- seed + 2,
// s2 <- seed + 3 (d each), and the d x b sketch p (64-byte aligned, owned).
// `seed` is kept as well: the library's calls are keyed by it.
template <typename Hash>
class matmul_sketch {
 public:
  matmul_sketch(int d, int b, uint64_t seed)
      : d(d), b(b), seed(seed), mod_mask(~(~UINT32_C(0) << detail::ilog2((uint32_t)b))),
        h1(Hash::draw(d, b, seed)), h2(Hash::draw(d, b, seed + 1)), s1(Hash::draw(d, b, seed + 2)),
        s2(Hash::draw(d, b, seed + 3)), p(alloc(d, b), &release) {}
  matmul_sketch(const matmul_sketch& o)
      : d(o.d), b(o.b), seed(o.seed), mod_mask(o.mod_mask), h1(o.h1), h2(o.h2), s1(o.s1), s2(o.s2),
        p(alloc(o.d, o.b), &release) {
    std::memcpy(p.get(), o.p.get(), sizeof(double) * (size_t)d * (size_t)b);
  }
  matmul_sketch(matmul_sketch&& o) noexcept
      : d(o.d), b(o.b), seed(o.seed), mod_mask(o.mod_mask), h1(std::move(o.h1)), h2(std::move(o.h2)),
        s1(std::move(o.s1)), s2(std::move(o.s2)), p(std::move(o.p)) {}
  matmul_sketch& operator=(const matmul_sketch& o) {
    if (this != &o) {
      matmul_sketch c(o);
      swap(c);
    }
    return *this;
  }
  matmul_sketch& operator=(matmul_sketch&& o) noexcept {
    if (this != &o) swap(o);
    return *this;
  }

  int d;
  int b;
  uint64_t seed;
  uint32_t mod_mask;  // x & mod_mask == x % b
  std::vector<Hash> h1, h2, s1, s2;
  std::unique_ptr<double, void (*)(double*)> p;

 private:
  static double* alloc(int d, int b) {
    const size_t n = (size_t)(d > 0 ? d : 0) * (size_t)(b > 0 ? b : 0);
    void* q = std::aligned_alloc(64, ((n * sizeof(double) + 63) / 64) * 64 + 64);
    if (!q) throw std::bad_alloc();
    std::memset(q, 0, n * sizeof(double));
    return static_cast<double*>(q);
  }
  static void release(double* q) { std::free(q); }
  void swap(matmul_sketch& o) noexcept {
    std::swap(d, o.d);
    std::swap(b, o.b);
    std::swap(seed, o.seed);
    std::swap(mod_mask, o.mod_mask);
    std::swap(h1, o.h1);
    std::swap(h2, o.h2);
    std::swap(s1, o.s1);
    std::swap(s2, o.s2);
    std::swap(p, o.p);
  }
};

template <typename Hash>
using matmul_fft_sketch = matmul_sketch<Hash>;
template <typename Hash>
using matmul_fwht_sketch = matmul_sketch<Hash>;

namespace detail {
// matmul_fft.hpp:29-33: without a seed, rng()() draws one; the sketch's
// functions are drawn from it, then the device fills p
template <typename Hash>
matmul_sketch<Hash> compressed(int variant, int64_t n_a, int64_t n_inner, int64_t n_b,
                               const double* A, const double* B, int d, int b,
                               std::optional<uint64_t> seed) {
  if (!seed) seed = rng()();
  matmul_sketch<Hash> s(d, b, *seed);
  throw_status(cmm_compressed_product(variant, Hash::kind, n_a, n_inner, n_b, A, B, d, b, 1, *seed,
                                      s.p.get(), nullptr));
  return s;
}

template <typename Hash>
void decompress(int variant, int cols, double* C, uint32_t i, uint32_t j,
                const matmul_sketch<Hash>& sk, double* /*scratch*/) {
  double out = 0.0;
  throw_status(cmm_decompress(variant, Hash::kind, sk.d, sk.b, sk.seed, sk.p.get(), 1, &i, &j, &out));
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
                              sketch.p.get(), count, i, j, out));
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
