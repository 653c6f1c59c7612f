// ref_capi.cpp -- a C entry layer over the reference's OWN headers
// (matmul_fft.hpp, matmul_fwht.hpp, hashing.hpp, rng.hpp, array.hpp,
// transform.hpp), compiled unchanged from the reference tree against the
// project shims in oracle/shims (FFTW3 / FXT / CBLAS are not installed).
// TEST INFRASTRUCTURE: used to cross-check the C restatement, to generate
// golden fixtures, and as the timed CPU baseline.  The product never loads it.
//
// Build: oracle/Makefile (target `ref`), output only into oracle/_ref/.
#include "matmul_fft.hpp"
#include "matmul_fwht.hpp"
#include "hashing.hpp"
#include "array.hpp"
#include "rng.hpp"

#include <omp.h>
#include <cstdint>
#include <cstring>

using namespace compmatmul;

namespace {
using tab8 = tabulation_hash<8, uint32_t, uint32_t>;
using tab16 = tabulation_hash<16, uint32_t, uint32_t>;

template <typename F>
int dispatch(int kind, F&& f) {
  switch (kind) {
    case 0: f((multiply_shift_hash*)nullptr); return 0;
    case 1: f((multiply_add_shift_hash*)nullptr); return 0;
    case 2: f((tab8*)nullptr); return 0;
    case 3: f((tab16*)nullptr); return 0;
  }
  return 1;
}
}  // namespace

extern "C" {

int ref_num_threads(void) { return omp_get_max_threads(); }

// matmul_fft<H> / matmul_fwht<H> (matmul_fft.hpp:156, matmul_fwht.hpp:145)
int ref_matmul(int variant, int kind, int n_a, int n_inner, int n_b, double* C, const double* AT,
               const double* B, int d, int b, uint64_t seed) {
  return dispatch(kind, [&](auto* tag) {
    using H = std::remove_pointer_t<decltype(tag)>;
    if (variant == 0) matmul_fft<H>(n_a, n_inner, n_b, C, AT, B, d, b, seed);
    else matmul_fwht<H>(n_a, n_inner, n_b, C, AT, B, d, b, seed);
  });
}

// matmul_compressed_product_{fft,fwht}<H> (matmul_fft.hpp:26, matmul_fwht.hpp:26)
int ref_compressed_product(int variant, int kind, int n_a, int n_inner, int n_b, const double* AT,
                           const double* B, int d, int b, uint64_t seed, double* p_out) {
  return dispatch(kind, [&](auto* tag) {
    using H = std::remove_pointer_t<decltype(tag)>;
    if (variant == 0) {
      auto s = matmul_compressed_product_fft<H>(n_a, n_inner, n_b, AT, B, d, b, seed);
      std::memcpy(p_out, s.p.get(), sizeof(double) * d * b);
    } else {
      auto s = matmul_compressed_product_fwht<H>(n_a, n_inner, n_b, AT, B, d, b, seed);
      std::memcpy(p_out, s.p.get(), sizeof(double) * d * b);
    }
  });
}

// Rows [i0,i1) of dense C from a sketch p (matmul_decompress_{fft,fwht},
// matmul_fft.hpp:136, matmul_fwht.hpp:123), OpenMP over rows as in
// matmul_fft.hpp:165-177.
int ref_decompress_rows(int variant, int kind, int d, int b, uint64_t seed, const double* p,
                        int n_b, int i0, int i1, double* C) {
  return dispatch(kind, [&](auto* tag) {
    using H = std::remove_pointer_t<decltype(tag)>;
    matmul_sketch<H> sketch(d, b, seed);
    std::memcpy(sketch.p.get(), p, sizeof(double) * d * b);
#pragma omp parallel
    {
      double* scratch = array::allocate<double>(d);
#pragma omp for schedule(guided)
      for (int i = i0; i < i1; ++i)
        for (int j = 0; j < n_b; ++j) {
          if (variant == 0) matmul_decompress_fft<H>(n_b, C, i, j, sketch, scratch);
          else matmul_decompress_fwht<H>(n_b, C, i, j, sketch, scratch);
        }
      array::deallocate(scratch);
    }
  });
}

// Bucket and sign of key under function `t` of the family drawn with
// (d, b, seed) -- hashing.hpp draw + operator() + sign.
int ref_hash_codes(int kind, int d, int b, uint64_t seed, int n, uint32_t* buckets, int* signs) {
  return dispatch(kind, [&](auto* tag) {
    using H = std::remove_pointer_t<decltype(tag)>;
    auto fns = H::draw(d, b, seed);
    for (int t = 0; t < d; ++t)
      for (int i = 0; i < n; ++i) {
        buckets[(size_t)t * n + i] = fns[t]((uint32_t)i);
        signs[(size_t)t * n + i] = fns[t].sign((uint32_t)i);
      }
  });
}

void ref_gemm(int n_a, int n_inner, int n_b, double* C, const double* AT, const double* B) {
  array::matmul_gemm<double>(n_a, n_inner, n_b, C, AT, B);
}

// transform.hpp fft_transformer / fwht_transformer, for the golden vectors
void ref_fft_fwd(int n, const double* x, double* X) {
  fft_transformer f(n);
  f.fwd(reinterpret_cast<std::complex<double>*>(X), x);
}
void ref_fft_inv(int n, const double* X, double* x) {
  fft_transformer f(n);
  f.inv(x, reinterpret_cast<const std::complex<double>*>(X));
}
void ref_fwht_fwd(int n, double* x) {
  fwht_transformer f(n);
  f.fwd(x);
}

uint64_t ref_rng_first(uint64_t seed) { return rng(seed)(); }
}
