// The reference's small exact products (tests.cpp:842-942, 1052-1150,
// 722-750) driven through the C++ header entry points of
// include/compmatmul_b200.hpp.  Exit status 0 on success.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "compmatmul_b200.hpp"

using namespace compmatmul_b200;

static const double AT_4x4[16] = {1, 5, 9, 13, 2, 6, 10, 14, 3, 7, 11, 15, 4, 8, 12, 16};
static const double AT_2x4[8] = {1, 3, 5, 7, 2, 4, 6, 8};
static const double AT_4x2[8] = {1, 5, 2, 6, 3, 7, 4, 8};
static const double B_4x4[16] = {17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32};
static const double B_2x4[8] = {9, 10, 11, 12, 13, 14, 15, 16};
static const double B_4x2[8] = {9, 10, 11, 12, 13, 14, 15, 16};
static const double B_4x8[32] = {1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16,
                                 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32};
static const double C_4x4x4[16] = {250, 260, 270, 280, 618, 644, 670, 696,
                                   986, 1028, 1070, 1112, 1354, 1412, 1470, 1528};
static const double C_4x2x4[16] = {35, 38, 41, 44, 79, 86, 93, 100, 123, 134, 145, 156, 167, 182, 197, 212};
static const double C_2x4x2[4] = {130, 140, 322, 348};
static const double C_2x4x8[16] = {170, 180, 190, 200, 210, 220, 230, 240,
                                   378, 404, 430, 456, 482, 508, 534, 560};

static int failures = 0;
static void check(bool ok, const char* what, int d, int b) {
  if (!ok) {
    std::printf("FAIL %s d=%d b=%d\n", what, d, b);
    ++failures;
  }
}
static bool near(int n, const double* a, const double* b, double tol) {
  for (int i = 0; i < n; ++i)
    if (std::fabs(a[i] - b[i]) > tol) return false;
  return true;
}

int main() {
  struct Case { const double *AT, *B, *C; int n_a, n_inner, n_b; };
  const Case cases[] = {{AT_4x4, B_4x4, C_4x4x4, 4, 4, 4}, {AT_2x4, B_2x4, C_4x2x4, 4, 2, 4},
                        {AT_4x2, B_4x2, C_2x4x2, 2, 4, 2}, {AT_4x2, B_4x8, C_2x4x8, 2, 4, 8}};
  const uint64_t seed = 25926;
  std::vector<double> C(64);
  const int fft_db[][2] = {{1, 2}, {1, 8}, {1, 32}, {3, 2}, {3, 8}, {5, 32}};
  const int fwht_db[][2] = {{1, 2}, {1, 8}, {1, 32}, {3, 2}, {3, 8}, {7, 32}};
  for (auto& db : fft_db) {
    const int d = db[0], b = db[1];
    auto sk = matmul_compressed_product_fft<multiply_add_shift_hash>(4, 4, 4, AT_4x4, B_4x4, d, b, seed);
    check(sk.seed == seed && (int)sk.p.size() == d * b, "fft sketch shape", d, b);
    std::vector<double> Cd(16), scratch(d);
    for (uint32_t i = 0; i < 4; ++i)
      for (uint32_t j = 0; j < 4; ++j) matmul_decompress_fft(4, Cd.data(), i, j, sk, scratch.data());
    if (d > 1 && b >= 32) {
      check(near(16, Cd.data(), C_4x4x4, 1e-6), "fft decompress", d, b);
      for (const Case& c : cases) {
        matmul_fft<multiply_add_shift_hash>(c.n_a, c.n_inner, c.n_b, C.data(), c.AT, c.B, d, b, seed);
        check(near(c.n_a * c.n_b, C.data(), c.C, 1e-6), "matmul_fft", d, b);
      }
    }
  }
  for (auto& db : fwht_db) {
    const int d = db[0], b = db[1];
    auto sk = matmul_compressed_product_fwht<multiply_add_shift_hash>(4, 4, 4, AT_4x4, B_4x4, d, b, seed);
    std::vector<double> Cd(16), scratch(d);
    for (uint32_t i = 0; i < 4; ++i)
      for (uint32_t j = 0; j < 4; ++j) matmul_decompress_fwht(4, Cd.data(), i, j, sk, scratch.data());
    if (d > 1 && b >= 32) {
      check(near(16, Cd.data(), C_4x4x4, 0.0), "fwht decompress (exact)", d, b);
      for (const Case& c : cases) {
        matmul_fwht<multiply_add_shift_hash>(c.n_a, c.n_inner, c.n_b, C.data(), c.AT, c.B, d, b, seed);
        check(near(c.n_a * c.n_b, C.data(), c.C, 0.0), "matmul_fwht (exact)", d, b);
      }
    }
  }
  for (const Case& c : cases) {
    array::matmul_gemm<double>(c.n_a, c.n_inner, c.n_b, C.data(), c.AT, c.B);
    check(near(c.n_a * c.n_b, C.data(), c.C, 0.0), "gemm (exact)", 0, 0);
  }
  // the other hash families go through the same entry points
  matmul_fft<multiply_shift_hash>(4, 4, 4, C.data(), AT_4x4, B_4x4, 5, 1024, 7);
  check(near(16, C.data(), C_4x4x4, 1e-6), "matmul_fft multiply_shift", 5, 1024);
  matmul_fwht<tabulation_hash<8, uint32_t, uint32_t>>(4, 4, 4, C.data(), AT_4x4, B_4x4, 5, 1024, 7);
  check(near(16, C.data(), C_4x4x4, 0.0), "matmul_fwht tabulation8", 5, 1024);
  matmul_fwht<tabulation_hash<16, uint32_t, uint32_t>>(4, 4, 4, C.data(), AT_4x4, B_4x4, 5, 1024, 7);
  check(near(16, C.data(), C_4x4x4, 0.0), "matmul_fwht tabulation16", 5, 1024);
  // reference exception types
  bool threw = false;
  try {
    matmul_fft<multiply_add_shift_hash>(4, 4, 4, C.data(), AT_4x4, B_4x4, 1, 12, 7);
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  check(threw, "invalid b throws std::invalid_argument", 1, 12);
  std::printf(failures ? "FAILED %d\n" : "ok\n", failures);
  return failures ? 1 : 0;
}
