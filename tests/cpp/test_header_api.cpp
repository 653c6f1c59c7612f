// The reference's own C++ unit cases, compiled against the drop-in header
// include/compmatmul_b200.hpp instead of the reference headers:
//   hash families and sign hashes      tests.cpp:146-461
//   sketch parameters (matmul_sketch)  tests.cpp:797-840
//   products through the sketch type   tests.cpp:842-942 (FFT), 1052-1150 (FWHT)
//   four hash families vs exact gemm   tests.cpp:944-1003, 1152-1211
//   gemm                               tests.cpp:722-750
// Argument "hash" runs only the host-side parts (no GPU needed); no
// argument runs everything.  Exit status 0 on success, and "ok" printed.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
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
#define REQUIRE(cond)                                                  \
  do {                                                                 \
    if (!(cond)) {                                                     \
      std::printf("FAIL line %d: %s\n", __LINE__, #cond);              \
      ++failures;                                                      \
    }                                                                  \
  } while (0)

static bool near(int n, const double* a, const double* b, double tol) {
  for (int i = 0; i < n; ++i)
    if (std::fabs(a[i] - b[i]) > tol) return false;
  return true;
}

// xoshiro256+ doubles (the reference test suite's drng, rng.hpp:81-110),
// used only to make the test inputs of tests.cpp:960-966
class test_drng {
 public:
  explicit test_drng(uint64_t seed) { cmm_rng_seed(seed, s_); }
  double operator()() {
    const uint64_t r = s_[0] + s_[3];
    const uint64_t t = s_[1] << 17;
    s_[2] ^= s_[0];
    s_[3] ^= s_[1];
    s_[1] ^= s_[2];
    s_[0] ^= s_[3];
    s_[2] ^= t;
    s_[3] = (s_[3] << 45) | (s_[3] >> 19);
    return (double)(r >> 11) * 0x1.0p-53;
  }

 private:
  uint64_t s_[4];
};

// ------------------------------------------------------------ host side
static void hash_cases() {
  // tests.cpp:90-96: the rng stream
  {
    rng r(1234);
    REQUIRE(r() == 0x0bab45d9a0e3ae53ULL);
    REQUIRE(r() == 0xd7c640660c19433eULL);
    REQUIRE(r() == 0xb0dedaa0d09a6691ULL);
    REQUIRE(r() == 0xdec9f41b58ec86ebULL);
  }
  // tests.cpp:146-222 multiply-shift
  {
    uint64_t seed = 123456;
    const uint32_t m = 64;
    const uint64_t a = 2749059519329956733ULL;
    multiply_shift_hash msh1(m, a);
    multiply_shift_hash msh2 = multiply_shift_hash::draw_one(m, seed);
    multiply_shift_hash msh3 = multiply_shift_hash::draw(1, m, seed)[0];
    int counts[64] = {0};
    for (uint32_t i = 0; i <= 128; ++i) {
      const uint32_t h = (uint32_t)((a * i) >> 58);
      REQUIRE(h == msh1(i));
      REQUIRE(h == msh2(i));
      REQUIRE(h == msh3(i));
      ++counts[h];
    }
    for (int i = 0; i < 64; ++i) REQUIRE(counts[i] > 0);
    auto sign = sign_hash<multiply_shift_hash>::draw_one(seed);
    for (uint32_t i = 0; i <= 128; ++i) {
      const int want = ((a * i) >> 63) == 1 ? 1 : -1;
      REQUIRE(sign(i) == want);
      REQUIRE(msh1.sign(i) == want);
    }
    const uint64_t a1 = 3688180003657674949ULL, a2 = 11729574476469721337ULL;
    seed = 19850;
    auto mshs = multiply_shift_hash::draw(2, 32, seed);
    auto signs1 = sign_hash<multiply_shift_hash>::draw(2, seed);
    auto signs2 = multiply_shift_hash::draw(2, 2, seed);
    for (uint32_t i = 0; i <= 1024; ++i) {
      REQUIRE(mshs[0](i) == (uint32_t)((a1 * i) >> 59));
      REQUIRE(mshs[1](i) == (uint32_t)((a2 * i) >> 59));
      const int w1 = ((a1 * i) >> 63) == 1 ? 1 : -1, w2 = ((a2 * i) >> 63) == 1 ? 1 : -1;
      REQUIRE(signs1[0](i) == w1);
      REQUIRE(signs1[1](i) == w2);
      REQUIRE(signs2[0].sign(i) == w1);
      REQUIRE(signs2[1].sign(i) == w2);
    }
  }
  // tests.cpp:226-311 multiply-add-shift
  {
    uint64_t seed = 123456;
    const uint32_t m = 128;
    const uint64_t a = 2366053268901514180ULL, b = 2749059519329956733ULL;
    multiply_add_shift_hash mash1(m, a, b);
    multiply_add_shift_hash mash2 = multiply_add_shift_hash::draw_one(m, seed);
    multiply_add_shift_hash mash3 = multiply_add_shift_hash::draw(1, m, seed)[0];
    for (uint32_t i = 0; i <= 512; ++i) {
      const uint32_t h = (uint32_t)((a * i + b) >> 57);
      REQUIRE(h == mash1(i));
      REQUIRE(h == mash2(i));
      REQUIRE(h == mash3(i));
    }
    auto sign = sign_hash<multiply_add_shift_hash>::draw_one(seed);
    for (uint32_t i = 0; i <= 512; ++i) {
      const int want = ((a * i + b) >> 63) == 1 ? 1 : -1;
      REQUIRE(sign(i) == want);
      REQUIRE(mash1.sign(i) == want);
    }
    seed = 22201;
    const uint64_t a1 = 2016826348251915964ULL, b1 = 17696970887482165528ULL;
    const uint64_t a2 = 6666994550483350943ULL, b2 = 1097363203091539945ULL;
    auto mashes = multiply_add_shift_hash::draw(2, 128, seed);
    auto signs = sign_hash<multiply_add_shift_hash>::draw(2, seed);
    for (uint32_t i = 0; i <= 2048; ++i) {
      REQUIRE(mashes[0](i) == (uint32_t)((a1 * i + b1) >> 57));
      REQUIRE(mashes[1](i) == (uint32_t)((a2 * i + b2) >> 57));
      const int w1 = ((a1 * i + b1) >> 63) == 1 ? 1 : -1, w2 = ((a2 * i + b2) >> 63) == 1 ? 1 : -1;
      REQUIRE(signs[0](i) == w1);
      REQUIRE(signs[1](i) == w2);
      REQUIRE(mashes[0].sign(i) == w1);
      REQUIRE(mashes[1].sign(i) == w2);
    }
  }
  // tests.cpp:315-455 tabulation over 8- and 16-bit characters
  {
    using T8 = tabulation_hash<8, uint32_t, uint32_t>;
    using T16 = tabulation_hash<16, uint32_t, uint32_t>;
    uint64_t seed = 23711;
    const uint32_t m = 256;
    rng prng(seed);
    std::vector<uint32_t> T1(4 * 256);
    for (auto& v : T1) v = (uint32_t)prng();
    T8 th8_1(m, T1.data());
    T8 th8_2 = T8::draw_one(m, seed);
    T8 th8_3 = T8::draw(1, m, seed)[0];
    auto tab8 = [&](const std::vector<uint32_t>& T, uint32_t x) {
      return T[x & 0xff] ^ T[256 + ((x >> 8) & 0xff)] ^ T[512 + ((x >> 16) & 0xff)] ^ T[768 + ((x >> 24) & 0xff)];
    };
    for (int i = 0; i < 256; ++i) {
      const uint32_t x = (uint32_t)prng();
      const uint32_t h = tab8(T1, x) >> 24;
      REQUIRE(h == th8_1(x));
      REQUIRE(h == th8_2(x));
      REQUIRE(h == th8_3(x));
    }
    auto th8_s = sign_hash<T8>::draw_one(seed);
    for (int i = 0; i < 256; ++i) {
      const uint32_t x = (uint32_t)prng();
      const int h1 = 2 * (int)(tab8(T1, x) >> 31) - 1;
      REQUIRE(h1 == th8_s(x));
      REQUIRE(h1 == th8_1.sign(x));
    }
    ++seed;
    prng = rng(seed);
    std::vector<uint32_t> T2(2 * 65536);
    for (auto& v : T2) v = (uint32_t)prng();
    auto tab16 = [&](const std::vector<uint32_t>& T, uint32_t x) { return T[x & 0xffff] ^ T[65536 + (x >> 16)]; };
    T16 th16_1(m, T2.data());
    T16 th16_2 = T16::draw_one(m, seed);
    T16 th16_3 = T16::draw(1, m, seed)[0];
    for (int i = 0; i < 256; ++i) {
      const uint32_t x = (uint32_t)prng();
      const uint32_t h = tab16(T2, x) >> 24;
      REQUIRE(h == th16_1(x));
      REQUIRE(h == th16_2(x));
      REQUIRE(h == th16_3(x));
    }
    auto th16_s = sign_hash<T16>::draw_one(seed);
    for (int i = 0; i < 256; ++i) {
      const uint32_t x = (uint32_t)prng();
      const int h1 = 2 * (int)(tab16(T2, x) >> 31) - 1;
      REQUIRE(h1 == th16_s(x));
      REQUIRE(h1 == th16_1.sign(x));
    }
    seed = 16321;
    prng = rng(seed);
    std::vector<uint32_t> T1a(1024), T1b(1024);
    for (auto& v : T1a) v = (uint32_t)prng();
    for (auto& v : T1b) v = (uint32_t)prng();
    auto t8s = T8::draw(2, 128, seed);
    auto th8_ss = sign_hash<T8>::draw(2, seed);
    for (int i = 0; i < 1024; ++i) {
      const uint32_t x = (uint32_t)prng();
      REQUIRE(t8s[0](x) == tab8(T1a, x) >> 25);
      REQUIRE(t8s[1](x) == tab8(T1b, x) >> 25);
    }
    for (int i = 0; i < 1024; ++i) {
      const uint32_t x = (uint32_t)prng();
      const int h1 = 2 * (int)(tab8(T1a, x) >> 31) - 1, h2 = 2 * (int)(tab8(T1b, x) >> 31) - 1;
      REQUIRE(th8_ss[0](x) == h1);
      REQUIRE(th8_ss[1](x) == h2);
      REQUIRE(t8s[0].sign(x) == h1);
      REQUIRE(t8s[1].sign(x) == h2);
    }
    ++seed;
    prng = rng(seed);
    std::vector<uint32_t> T2a(2 * 65536), T2b(2 * 65536);
    for (auto& v : T2a) v = (uint32_t)prng();
    for (auto& v : T2b) v = (uint32_t)prng();
    auto t16s = T16::draw(2, 128, seed);
    auto th16_ss = sign_hash<T16>::draw(2, seed);
    for (int i = 0; i < 1024; ++i) {
      const uint32_t x = (uint32_t)prng();
      REQUIRE(t16s[0](x) == tab16(T2a, x) >> 25);
      REQUIRE(t16s[1](x) == tab16(T2b, x) >> 25);
    }
    for (int i = 0; i < 1024; ++i) {
      const uint32_t x = (uint32_t)prng();
      const int h1 = 2 * (int)(tab16(T2a, x) >> 31) - 1, h2 = 2 * (int)(tab16(T2b, x) >> 31) - 1;
      REQUIRE(th16_ss[0](x) == h1);
      REQUIRE(th16_ss[1](x) == h2);
      REQUIRE(t16s[0].sign(x) == h1);
      REQUIRE(t16s[1].sign(x) == h2);
    }
  }
  // tests.cpp:797-840: multiply-add-shift draws and the sketch's functions
  {
    multiply_add_shift_hash h = multiply_add_shift_hash::draw_one(32, 8876);
    const uint64_t a = 15506110424104283675ULL, b = 3138147583905456810ULL;
    REQUIRE(h.get_a() == a);
    REQUIRE(h.get_b() == b);
    rng r(32149);
    for (int i = 0; i < 100; ++i) {
      const uint32_t x = (uint32_t)r();
      const uint32_t hash = (uint32_t)((a * x + b) >> 59);
      REQUIRE(h(x) == hash);
      REQUIRE(h.sign(x) == ((hash >> 4) ? 1 : -1));
    }
    matmul_fft_sketch<multiply_add_shift_hash> sketch(2, 2, 3483);
    REQUIRE(sketch.h1.size() == 2);
    REQUIRE(sketch.h1[0].get_a() == 1312110179027324775ULL);
    REQUIRE(sketch.h1[0].get_b() == 15465668779316680995ULL);
    REQUIRE(sketch.h1[1].get_a() == 4555306672462241870ULL);
    REQUIRE(sketch.h1[1].get_b() == 12288159137770073612ULL);
    REQUIRE(sketch.h2.size() == 2);
    REQUIRE(sketch.h2[0].get_a() == 4329212686603688483ULL);
    REQUIRE(sketch.h2[0].get_b() == 10307990599335447505ULL);
    REQUIRE(sketch.h2[1].get_a() == 12597734872139453857ULL);
    REQUIRE(sketch.h2[1].get_b() == 15119207240207437602ULL);
    REQUIRE(sketch.s1.size() == 2);
    REQUIRE(sketch.s1[0].get_a() == 11899074044546628492ULL);
    REQUIRE(sketch.s1[0].get_b() == 298345645907162146ULL);
    REQUIRE(sketch.s1[1].get_a() == 8628211646415106536ULL);
    REQUIRE(sketch.s1[1].get_b() == 12647867801867038929ULL);
    REQUIRE(sketch.s2.size() == 2);
    REQUIRE(sketch.s2[0].get_a() == 7008367753992221008ULL);
    REQUIRE(sketch.s2[0].get_b() == 16948937881964684143ULL);
    REQUIRE(sketch.s2[1].get_a() == 10319872211339334476ULL);
    REQUIRE(sketch.s2[1].get_b() == 13096518497071785733ULL);
    REQUIRE(sketch.d == 2 && sketch.b == 2 && sketch.mod_mask == 1u);
    REQUIRE(sketch.p.get() != nullptr && sketch.p.get()[0] == 0.0 && sketch.p.get()[3] == 0.0);
    // copies own their p; moves take it
    matmul_fft_sketch<multiply_add_shift_hash> copy(sketch);
    copy.p.get()[0] = 1.0;
    REQUIRE(sketch.p.get()[0] == 0.0 && copy.h1[1].get_a() == sketch.h1[1].get_a());
    matmul_fft_sketch<multiply_add_shift_hash> moved(std::move(copy));
    REQUIRE(moved.p.get()[0] == 1.0 && moved.b == 2);
    bool threw = false;
    try {
      matmul_fft_sketch<multiply_add_shift_hash> bad(2, 12, 1);
    } catch (const std::invalid_argument&) {
      threw = true;
    }
    REQUIRE(threw);
  }
}

// ------------------------------------------------------------- GPU side
template <bool FFT>
static void sketch_product_cases() {
  struct Case { const double *AT, *B, *C; int n_a, n_inner, n_b; };
  const Case cases[] = {{AT_4x4, B_4x4, C_4x4x4, 4, 4, 4}, {AT_2x4, B_2x4, C_4x2x4, 4, 2, 4},
                        {AT_4x2, B_4x2, C_2x4x2, 2, 4, 2}, {AT_4x2, B_4x8, C_2x4x8, 2, 4, 8}};
  const int db_fft[][2] = {{1, 2}, {1, 8}, {1, 32}, {3, 2}, {3, 8}, {5, 32}};
  const int db_fwht[][2] = {{1, 2}, {1, 8}, {1, 32}, {3, 2}, {3, 8}, {7, 32}};
  const uint64_t seed = 25926;
  // FWHT of integer inputs is exact; the FFT is within the reference's 1e-6
  const double tol = FFT ? 1e-6 : 0.0;
  for (int c = 0; c < 6; ++c) {
    const int d = FFT ? db_fft[c][0] : db_fwht[c][0], b = FFT ? db_fft[c][1] : db_fwht[c][1];
    matmul_sketch<multiply_add_shift_hash> sketch(d, b, seed);
    std::vector<uint64_t> ab;
    for (int i = 0; i < d; ++i)
      for (const auto* set : {&sketch.h1, &sketch.h2, &sketch.s1, &sketch.s2}) {
        ab.push_back((*set)[i].get_a());
        ab.push_back((*set)[i].get_b());
      }
    std::vector<double> C(16, 0.0), xs(d);
    sketch = FFT ? matmul_compressed_product_fft<multiply_add_shift_hash>(4, 4, 4, AT_4x4, B_4x4, d, b, seed)
                 : matmul_compressed_product_fwht<multiply_add_shift_hash>(4, 4, 4, AT_4x4, B_4x4, d, b, seed);
    size_t e = 0;
    for (int i = 0; i < d; ++i)
      for (const auto* set : {&sketch.h1, &sketch.h2, &sketch.s1, &sketch.s2}) {
        REQUIRE((*set)[i].get_a() == ab[e++]);
        REQUIRE((*set)[i].get_b() == ab[e++]);
      }
    for (uint32_t i = 0; i < 4; ++i)
      for (uint32_t j = 0; j < 4; ++j) {
        if (FFT) matmul_decompress_fft(4, C.data(), i, j, sketch, xs.data());
        else matmul_decompress_fwht(4, C.data(), i, j, sketch, xs.data());
      }
    if (d > 1 && b >= 32) {
      REQUIRE(near(16, C.data(), C_4x4x4, tol));
      for (const Case& k : cases) {
        std::vector<double> Ck(64, 0.0);
        if (FFT) matmul_fft<multiply_add_shift_hash>(k.n_a, k.n_inner, k.n_b, Ck.data(), k.AT, k.B, d, b, seed);
        else matmul_fwht<multiply_add_shift_hash>(k.n_a, k.n_inner, k.n_b, Ck.data(), k.AT, k.B, d, b, seed);
        REQUIRE(near(k.n_a * k.n_b, Ck.data(), k.C, tol));
      }
    }
  }
  // tests.cpp:944-1003 / 1152-1211: n = 16 random inputs, four hash
  // families against the exact product, 1e-12 absolute
  const uint64_t s2 = 15954;
  const int n = 16;
  std::vector<double> AT(n * n), B(n * n), C1(n * n), C2(n * n), C3(n * n), C4(n * n), C5(n * n);
  test_drng dr(s2);
  for (int i = 0; i < n * n; ++i) {
    AT[i] = dr();
    B[i] = dr();
  }
  array::matmul_gemm<double>(n, n, n, C1.data(), AT.data(), B.data());
  using T8 = tabulation_hash<8, uint32_t, uint32_t>;
  using T16 = tabulation_hash<16, uint32_t, uint32_t>;
  if (FFT) {
    matmul_fft<multiply_add_shift_hash>(n, n, n, C2.data(), AT.data(), B.data(), 5, 1024, s2 + 1);
    matmul_fft<multiply_shift_hash>(n, n, n, C3.data(), AT.data(), B.data(), 5, 1024, s2 + 2);
    matmul_fft<T8>(n, n, n, C4.data(), AT.data(), B.data(), 11, 2048, s2 + 3);
    matmul_fft<T16>(n, n, n, C5.data(), AT.data(), B.data(), 11, 1024, s2 + 4);
  } else {
    matmul_fwht<multiply_add_shift_hash>(n, n, n, C2.data(), AT.data(), B.data(), 5, 2048, s2 + 1);
    matmul_fwht<multiply_shift_hash>(n, n, n, C3.data(), AT.data(), B.data(), 5, 2048, s2 + 2);
    matmul_fwht<T8>(n, n, n, C4.data(), AT.data(), B.data(), 11, 2048, s2 + 3);
    matmul_fwht<T16>(n, n, n, C5.data(), AT.data(), B.data(), 11, 1024, s2 + 4);
  }
  REQUIRE(near(n * n, C1.data(), C2.data(), 1e-12));
  REQUIRE(near(n * n, C1.data(), C3.data(), 1e-12));
  REQUIRE(near(n * n, C1.data(), C4.data(), 1e-12));
  REQUIRE(near(n * n, C1.data(), C5.data(), 1e-12));
}

static void device_cases() {
  sketch_product_cases<true>();
  sketch_product_cases<false>();
  // tests.cpp:722-750: exact gemm
  struct Case { const double *AT, *B, *C; int n_a, n_inner, n_b; };
  const Case cases[] = {{AT_4x4, B_4x4, C_4x4x4, 4, 4, 4}, {AT_2x4, B_2x4, C_4x2x4, 4, 2, 4},
                        {AT_4x2, B_4x2, C_2x4x2, 2, 4, 2}, {AT_4x2, B_4x8, C_2x4x8, 2, 4, 8}};
  for (const Case& c : cases) {
    std::vector<double> C(64);
    array::matmul_gemm<double>(c.n_a, c.n_inner, c.n_b, C.data(), c.AT, c.B);
    REQUIRE(near(c.n_a * c.n_b, C.data(), c.C, 0.0));
  }
  // a sketch without a seed draws one from the clock, as rng()() does
  auto sk = matmul_compressed_product_fft<multiply_add_shift_hash>(4, 4, 4, AT_4x4, B_4x4, 5, 1024);
  std::vector<double> C(16), xs(5);
  for (uint32_t i = 0; i < 4; ++i)
    for (uint32_t j = 0; j < 4; ++j) matmul_decompress_fft(4, C.data(), i, j, sk, xs.data());
  REQUIRE(near(16, C.data(), C_4x4x4, 1e-6));
  // batched listed-entry queries on the same sketch
  const uint32_t qi[3] = {0, 3, 2}, qj[3] = {1, 3, 0};
  double qv[3];
  decompress_entries(CMM_VARIANT_FFT, sk, 3, qi, qj, qv);
  REQUIRE(std::fabs(qv[0] - 260) < 1e-6 && std::fabs(qv[1] - 1528) < 1e-6 && std::fabs(qv[2] - 986) < 1e-6);
  // reference exception types
  bool threw = false;
  try {
    matmul_fft<multiply_add_shift_hash>(4, 4, 4, C.data(), AT_4x4, B_4x4, 1, 12, 7);
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  REQUIRE(threw);
}

int main(int argc, char** argv) {
  const bool host_only = argc > 1 && std::strcmp(argv[1], "hash") == 0;
  hash_cases();
  if (!host_only) device_cases();
  std::printf(failures ? "FAILED %d\n" : "ok\n", failures);
  return failures ? 1 : 0;
}
