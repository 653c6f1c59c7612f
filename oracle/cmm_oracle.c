/*
 * cmm_oracle.c -- CPU restatement of the compressed matrix multiplication
 * path of mkarppa/compmatmul.  TEST INFRASTRUCTURE ONLY: this file is the
 * checker that the CUDA path is compared against.  Only tests/, the smoke
 * check and bench.py's CPU-baseline leg load it; the product never does.
 *
 * Plain C99, FP64.  The independent repetitions of the compressed product
 * and the rows of the decompression run on OpenMP threads, with every sum
 * in the reference's order, so results do not depend on the thread count.
 * Every function names the reference file:line it restates.  Parity of this restatement is pinned by the
 * reference's own golden vectors (tests.cpp / test.py constants, see
 * tests/test_oracle_golden.py) and by cross-checks against the reference
 * headers compiled with project shims (oracle/_ref, see oracle/Makefile).
 *
 * Conventions (matmul_fft.hpp:19-24):
 *   AT is n_inner x n_a row-major (row k of AT = column k of A),
 *   B  is n_inner x n_b row-major, C = A^T B ... i.e. C[i][j] =
 *   sum_k AT[k][i] * B[k][j], C is n_a x n_b row-major.
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CMO_MS 0    /* multiply-shift            hashing.hpp:27-102  */
#define CMO_MAS 1   /* multiply-add-shift        hashing.hpp:111-183 */
#define CMO_TAB8 2  /* simple tabulation, 8-bit  hashing.hpp:232-320 */
#define CMO_TAB16 3 /* simple tabulation, 16-bit hashing.hpp:232-320 */

#define CMO_FFT 0
#define CMO_FWHT 1

/* ------------------------------------------------------------------ rng */

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* splitmix64 seeding of the 4-word state, rng.hpp:26-33 */
void cmo_rng_seed(uint64_t* s, uint64_t x) {
  for (int i = 0; i < 4; ++i) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    s[i] = z ^ (z >> 31);
  }
}

static void xoshiro_advance(uint64_t* s) {
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl64(s[3], 45);
}

/* xoshiro256** output, rng.hpp:59-72 */
uint64_t cmo_rng_next(uint64_t* s) {
  const uint64_t r = rotl64(s[1] * 5, 7) * 9;
  xoshiro_advance(s);
  return r;
}

/* xoshiro256+ double in [0,1), rng.hpp:94-107 */
double cmo_drng_next(uint64_t* s) {
  const uint64_t r = s[0] + s[3];
  xoshiro_advance(s);
  return (double)(r >> 11) * 0x1.0p-53;
}

/* ------------------------------------------------------------- hashing */

/* Bytes of parameters per hash function of each family. */
size_t cmo_hash_param_bytes(int kind) {
  switch (kind) {
    case CMO_MS: return 8;            /* a                      */
    case CMO_MAS: return 16;          /* a, b                   */
    case CMO_TAB8: return 4 * 256 * 4;   /* T[4][256]  u32      */
    case CMO_TAB16: return 2 * 65536 * 4; /* T[2][65536] u32    */
  }
  return 0;
}

/*
 * Draw n functions of one family from a single rng stream seeded with
 * `seed`: multiply_shift_hash::draw (hashing.hpp:69-87, odd `a` by
 * rejection), multiply_add_shift_hash::draw (hashing.hpp:145-160, a then b),
 * tabulation_hash::draw (hashing.hpp:277-295, table words truncated to u32
 * in T[c][v] row-major order).
 */
void cmo_hash_draw(int kind, int n, uint64_t seed, void* out) {
  uint64_t s[4];
  cmo_rng_seed(s, seed);
  if (kind == CMO_MS) {
    uint64_t* a = (uint64_t*)out;
    for (int f = 0; f < n; ++f) {
      uint64_t v;
      do { v = cmo_rng_next(s); } while ((v & 1) == 0);
      a[f] = v;
    }
  } else if (kind == CMO_MAS) {
    uint64_t* ab = (uint64_t*)out;
    for (int f = 0; f < n; ++f) {
      ab[2 * f] = cmo_rng_next(s);
      ab[2 * f + 1] = cmo_rng_next(s);
    }
  } else {
    size_t words = cmo_hash_param_bytes(kind) / 4;
    uint32_t* T = (uint32_t*)out;
    for (size_t w = 0; w < (size_t)n * words; ++w) T[w] = (uint32_t)cmo_rng_next(s);
  }
}

static int ilog2_u64(uint64_t x) {
  int r = -1;
  while (x) { ++r; x >>= 1; }
  return r;
}

/* The full pre-shift hash word: 64-bit for multiply families, 32-bit for
 * tabulation.  hashing.hpp:91-93, 163-165, 298-305. */
static uint64_t hash_word(int kind, const void* fn, uint32_t key) {
  if (kind == CMO_MS) {
    const uint64_t* a = (const uint64_t*)fn;
    return a[0] * (uint64_t)key;
  } else if (kind == CMO_MAS) {
    const uint64_t* ab = (const uint64_t*)fn;
    return ab[0] * (uint64_t)key + ab[1];
  } else if (kind == CMO_TAB8) {
    const uint32_t* T = (const uint32_t*)fn;
    uint32_t h = 0;
    for (int c = 0; c < 4; ++c) h ^= T[c * 256 + ((key >> (8 * c)) & 0xffu)];
    return h;
  } else {
    const uint32_t* T = (const uint32_t*)fn;
    return (uint32_t)(T[key & 0xffffu] ^ T[65536 + (key >> 16)]);
  }
}

/* Bucket in [0,b): word >> (64 - log2 b) or >> (32 - log2 b). */
uint32_t cmo_hash_bucket(int kind, const void* fn, int b, uint32_t key) {
  const int lg = ilog2_u64((uint64_t)b);
  const uint64_t w = hash_word(kind, fn, key);
  if (kind == CMO_MS || kind == CMO_MAS) return (uint32_t)(w >> (64 - lg));
  return (uint32_t)((uint32_t)w >> (32 - lg));
}

/* Sign from the top bit of the same word: +1 if set, -1 otherwise.
 * hashing.hpp:95-97, 167-169, 307-314. */
int cmo_hash_sign(int kind, const void* fn, uint32_t key) {
  const uint64_t w = hash_word(kind, fn, key);
  if (kind == CMO_MS || kind == CMO_MAS) return (w >> 63) ? 1 : -1;
  return ((uint32_t)w >> 31) ? 1 : -1;
}

/* ------------------------------------------------------------ transforms */

/* Twiddles of a length-n transform (n a power of two) with direction sign:
 * w[2j], w[2j+1] = cos, sin of the long double angle sign * 2 pi j / n, for
 * j < n/2.  Stage len of cfft reads entry j = k (n / len): its angle
 * sign * 2 pi k / len is the same long double value bit for bit (scaling
 * numerator and denominator by the power of two n / len commutes with
 * rounding), so the table changes no result; it only computes each
 * cosl / sinl once per (n, sign) instead of once per stage and k in every
 * call.  Tables are kept for the life of the process (guarded by a mutex:
 * ctypes callers may run on several threads). */
static pthread_mutex_t tw_mu = PTHREAD_MUTEX_INITIALIZER;
static double* tw_cache[2][32];
static const double* twiddle_table(int n, int sign) {
  int lg = 0;
  while ((1 << lg) < n) ++lg;
  const int si = sign > 0;
  pthread_mutex_lock(&tw_mu);
  if (!tw_cache[si][lg]) {
    const int h = n / 2 > 0 ? n / 2 : 1;
    double* w = (double*)malloc(sizeof(double) * 2 * (size_t)h);
    for (int j = 0; j < n / 2; ++j) {
      const long double ang = (long double)sign * 2.0L * 3.14159265358979323846264338327950288L * j / n;
      w[2 * j] = (double)cosl(ang);
      w[2 * j + 1] = (double)sinl(ang);
    }
    tw_cache[si][lg] = w;
  }
  const double* w = tw_cache[si][lg];
  pthread_mutex_unlock(&tw_mu);
  return w;
}

/* In-place iterative radix-2 complex DFT, sign -1 (forward) or +1
 * (inverse, unnormalised).  Twiddles from long double sin/cos
 * (twiddle_table). */
static void cfft(int n, double* re, double* im, int sign) {
  const double* tw = twiddle_table(n, sign);
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      double t = re[i]; re[i] = re[j]; re[j] = t;
      t = im[i]; im[i] = im[j]; im[j] = t;
    }
  }
  for (int len = 2; len <= n; len <<= 1) {
    const int half = len >> 1;
    const int step = n / len;
    /* every butterfly of a stage is independent: blocks outer, k inner
     * (contiguous), the same operations as any other order */
    for (int s = 0; s < n; s += len) {
      for (int k = 0; k < half; ++k) {
        const double wr = tw[2 * k * step], wi = tw[2 * k * step + 1];
        const int a = s + k, c = s + k + half;
        const double xr = re[c] * wr - im[c] * wi;
        const double xi = re[c] * wi + im[c] * wr;
        re[c] = re[a] - xr; im[c] = im[a] - xi;
        re[a] += xr; im[a] += xi;
      }
    }
  }
}

/* FFTW r2c semantics (transform.hpp:57-61): X[f] = sum_h x[h] e^{-2 pi i f h / n},
 * f = 0..n/2; X is interleaved (re,im) of length n/2+1. */
void cmo_fft_r2c(int n, const double* x, double* X) {
  double* re = (double*)malloc(sizeof(double) * n);
  double* im = (double*)calloc(n, sizeof(double));
  memcpy(re, x, sizeof(double) * n);
  cfft(n, re, im, -1);
  for (int f = 0; f <= n / 2; ++f) { X[2 * f] = re[f]; X[2 * f + 1] = im[f]; }
  free(re); free(im);
}

/* FFTW c2r semantics (transform.hpp:68-73 before the 1/n scaling):
 * x[h] = sum_f X[f] e^{+2 pi i f h / n} over the Hermitian extension;
 * the imaginary parts of X[0] and X[n/2] are ignored. */
void cmo_fft_c2r(int n, const double* X, double* x) {
  double* re = (double*)malloc(sizeof(double) * n);
  double* im = (double*)malloc(sizeof(double) * n);
  for (int f = 0; f <= n / 2; ++f) { re[f] = X[2 * f]; im[f] = X[2 * f + 1]; }
  im[0] = 0.0;
  if (n > 1) im[n / 2] = 0.0;
  for (int f = n / 2 + 1; f < n; ++f) { re[f] = X[2 * (n - f)]; im[f] = -X[2 * (n - f) + 1]; }
  cfft(n, re, im, +1);
  memcpy(x, re, sizeof(double) * n);
  free(re); free(im);
}

/* Natural (Sylvester / Walsh-Kronecker) order unnormalised WHT, in place;
 * the semantics of FXT walsh_wak used at transform.hpp:111,128. */
void cmo_fwht(int n, double* x) {
  for (int len = 1; len < n; len <<= 1)
    for (int s = 0; s < n; s += 2 * len)
      for (int k = s; k < s + len; ++k) {
        const double u = x[k], v = x[k + len];
        x[k] = u + v;
        x[k + len] = u - v;
      }
}

/* ------------------------------------------------------ sketch parameters */

/* The 4*d hash functions of a matmul_sketch (matmul_sketch.hpp:11-20):
 * h1 <- seed, h2 <- seed+1, s1 <- seed+2, s2 <- seed+3, each draw(d, b, .). */
typedef struct {
  int kind, d, b;
  unsigned char *h1, *h2, *s1, *s2;
  size_t fb; /* bytes per function */
} cmo_sketch_fns;

static void sketch_fns_init(cmo_sketch_fns* S, int kind, int d, int b, uint64_t seed) {
  S->kind = kind; S->d = d; S->b = b;
  S->fb = cmo_hash_param_bytes(kind);
  S->h1 = (unsigned char*)malloc(S->fb * d);
  S->h2 = (unsigned char*)malloc(S->fb * d);
  S->s1 = (unsigned char*)malloc(S->fb * d);
  S->s2 = (unsigned char*)malloc(S->fb * d);
  cmo_hash_draw(kind, d, seed + 0, S->h1);
  cmo_hash_draw(kind, d, seed + 1, S->h2);
  cmo_hash_draw(kind, d, seed + 2, S->s1);
  cmo_hash_draw(kind, d, seed + 3, S->s2);
}

static void sketch_fns_free(cmo_sketch_fns* S) {
  free(S->h1); free(S->h2); free(S->s1); free(S->s2);
}

/* Per-index bucket/sign codes of one side: code = bucket | (sign>0) << 31. */
void cmo_sketch_codes(int kind, int d, int b, uint64_t seed, int side, int64_t n, uint32_t* codes) {
  cmo_sketch_fns S;
  sketch_fns_init(&S, kind, d, b, seed);
  const unsigned char* H = side == 0 ? S.h1 : S.h2;
  const unsigned char* G = side == 0 ? S.s1 : S.s2;
  for (int t = 0; t < d; ++t)
    for (int64_t i = 0; i < n; ++i) {
      uint32_t h = cmo_hash_bucket(kind, H + S.fb * t, b, (uint32_t)i);
      int s = cmo_hash_sign(kind, G + S.fb * t, (uint32_t)i);
      codes[(size_t)t * n + i] = h | (s > 0 ? 0x80000000u : 0u);
    }
  sketch_fns_free(&S);
}

/* -------------------------------------------------- compressed product */

/*
 * matmul_compressed_product_fft (matmul_fft.hpp:25-129) and
 * matmul_compressed_product_fwht (matmul_fwht.hpp:25-114), serial.
 * p is d*b doubles (matmul_sketch::p).  Returns 0 on success.
 */
int cmo_compressed_product(int variant, int kind, int64_t n_a, int64_t n_inner, int64_t n_b,
                           const double* AT, const double* B, int d, int b, uint64_t seed,
                           double* p) {
  cmo_sketch_fns S;
  sketch_fns_init(&S, kind, d, b, seed);
  const int nc = b / 2 + 1;
  double* acc = (double*)calloc((size_t)d * (variant == CMO_FFT ? 2 * nc : b), sizeof(double));
  /* per-index codes: hash once per (t,i) instead of per (k,t,i); same values */
  uint32_t* hA = (uint32_t*)malloc(sizeof(uint32_t) * d * n_a);
  int8_t* sA = (int8_t*)malloc((size_t)d * n_a);
  uint32_t* hB = (uint32_t*)malloc(sizeof(uint32_t) * d * n_b);
  int8_t* sB = (int8_t*)malloc((size_t)d * n_b);
  for (int t = 0; t < d; ++t) {
    for (int64_t i = 0; i < n_a; ++i) {
      hA[t * n_a + i] = cmo_hash_bucket(kind, S.h1 + S.fb * t, b, (uint32_t)i);
      sA[t * n_a + i] = (int8_t)cmo_hash_sign(kind, S.s1 + S.fb * t, (uint32_t)i);
    }
    for (int64_t j = 0; j < n_b; ++j) {
      hB[t * n_b + j] = cmo_hash_bucket(kind, S.h2 + S.fb * t, b, (uint32_t)j);
      sB[t * n_b + j] = (int8_t)cmo_hash_sign(kind, S.s2 + S.fb * t, (uint32_t)j);
    }
  }
  /* The repetitions are independent and each accumulates over k in
   * ascending order, as the reference's k loop does for every t, so they
   * run on separate threads (OpenMP when built with it) with the same sums
   * in the same order: results do not depend on the thread count. */
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < d; ++t) {
    double* pa = (double*)malloc(sizeof(double) * b);
    double* pb = (double*)malloc(sizeof(double) * b);
    double* Xa = (double*)malloc(sizeof(double) * 2 * nc);
    double* Xb = (double*)malloc(sizeof(double) * 2 * nc);
    for (int64_t k = 0; k < n_inner; ++k) {
      const double* a = AT + (size_t)k * n_a;
      const double* bb = B + (size_t)k * n_b;
      memset(pa, 0, sizeof(double) * b);
      memset(pb, 0, sizeof(double) * b);
      /* matmul_fft.hpp:78-80 */
      for (int64_t i = 0; i < n_a; ++i) pa[hA[t * n_a + i]] += sA[t * n_a + i] * a[i];
      /* matmul_fft.hpp:89-91 */
      for (int64_t j = 0; j < n_b; ++j) pb[hB[t * n_b + j]] += sB[t * n_b + j] * bb[j];
      if (variant == CMO_FFT) {
        /* matmul_fft.hpp:95-106: r2c both, complex multiply, accumulate */
        cmo_fft_r2c(b, pa, Xa);
        cmo_fft_r2c(b, pb, Xb);
        double* P = acc + (size_t)t * 2 * nc;
        for (int f = 0; f < nc; ++f) {
          const double ar = Xa[2 * f], ai = Xa[2 * f + 1];
          const double br = Xb[2 * f], bi = Xb[2 * f + 1];
          P[2 * f] += ar * br - ai * bi;
          P[2 * f + 1] += ar * bi + ai * br;
        }
      } else {
        /* matmul_fwht.hpp:75,86,91-93 */
        cmo_fwht(b, pa);
        cmo_fwht(b, pb);
        double* P = acc + (size_t)t * b;
        for (int f = 0; f < b; ++f) P[f] += pa[f] * pb[f];
      }
    }
    free(pa); free(pb); free(Xa); free(Xb);
  }
  const double inv_b = 1.0 / b;
  for (int t = 0; t < d; ++t) {
    double* pt = p + (size_t)t * b;
    if (variant == CMO_FFT) {
      /* matmul_fft.hpp:118-121, transform.hpp:68-73 */
      cmo_fft_c2r(b, acc + (size_t)t * 2 * nc, pt);
    } else {
      /* matmul_fwht.hpp:101-108, transform.hpp:127-130 */
      memcpy(pt, acc + (size_t)t * b, sizeof(double) * b);
      cmo_fwht(b, pt);
    }
    for (int h = 0; h < b; ++h) pt[h] *= inv_b;
  }
  free(acc);
  free(hA); free(sA); free(hB); free(sB);
  sketch_fns_free(&S);
  return 0;
}

/* ----------------------------------------------------------- decompress */

/* array::median (array.hpp:323-328): element size/2 of ascending order. */
double cmo_median(int n, double* xs) {
  for (int i = 1; i < n; ++i) {
    double v = xs[i];
    int j = i - 1;
    while (j >= 0 && xs[j] > v) { xs[j + 1] = xs[j]; --j; }
    xs[j + 1] = v;
  }
  return xs[n / 2];
}

/*
 * Dense decompression, matmul_fft.hpp:135-147,165-177 (FFT index
 * (h1+h2) & (b-1)) and matmul_fwht.hpp:122-134,154-166 (index h1 ^ h2).
 * Rows [i0, i1) of C are written (C points at row 0).
 */
int cmo_decompress_rows(int variant, int kind, int d, int b, uint64_t seed, const double* p,
                        int64_t n_a, int64_t n_b, int64_t i0, int64_t i1, double* C) {
  (void)n_a;
  cmo_sketch_fns S;
  sketch_fns_init(&S, kind, d, b, seed);
  const uint32_t mask = (uint32_t)b - 1u;
  uint32_t* h2 = (uint32_t*)malloc(sizeof(uint32_t) * d * n_b);
  int8_t* s2 = (int8_t*)malloc((size_t)d * n_b);
  for (int t = 0; t < d; ++t)
    for (int64_t j = 0; j < n_b; ++j) {
      h2[t * n_b + j] = cmo_hash_bucket(kind, S.h2 + S.fb * t, b, (uint32_t)j);
      s2[t * n_b + j] = (int8_t)cmo_hash_sign(kind, S.s2 + S.fb * t, (uint32_t)j);
    }
  /* rows are independent (each entry is its own median): OpenMP threads
   * when built with it, each with its own scratch; the same values */
#pragma omp parallel
  {
    double* scratch = (double*)malloc(sizeof(double) * d);
    uint32_t* h1 = (uint32_t*)malloc(sizeof(uint32_t) * d);
    int* s1 = (int*)malloc(sizeof(int) * d);
#pragma omp for schedule(static)
    for (int64_t i = i0; i < i1; ++i) {
      for (int t = 0; t < d; ++t) {
        h1[t] = cmo_hash_bucket(kind, S.h1 + S.fb * t, b, (uint32_t)i);
        s1[t] = cmo_hash_sign(kind, S.s1 + S.fb * t, (uint32_t)i);
      }
      for (int64_t j = 0; j < n_b; ++j) {
        for (int t = 0; t < d; ++t) {
          const uint32_t hj = h2[t * n_b + j];
          const uint32_t h = variant == CMO_FFT ? ((h1[t] + hj) & mask) : (h1[t] ^ hj);
          const int s = s1[t] * s2[t * n_b + j];
          scratch[t] = s * p[(size_t)t * b + h];
        }
        C[(size_t)i * n_b + j] = cmo_median(d, scratch);
      }
    }
    free(scratch); free(h1); free(s1);
  }
  free(h2); free(s2);
  sketch_fns_free(&S);
  return 0;
}

/* matmul_fft / matmul_fwht drivers (matmul_fft.hpp:155-178,
 * matmul_fwht.hpp:144-167): compressed product + dense decompression. */
int cmo_matmul(int variant, int kind, int64_t n_a, int64_t n_inner, int64_t n_b, double* C,
               const double* AT, const double* B, int d, int b, uint64_t seed) {
  double* p = (double*)malloc(sizeof(double) * d * b);
  cmo_compressed_product(variant, kind, n_a, n_inner, n_b, AT, B, d, b, seed, p);
  cmo_decompress_rows(variant, kind, d, b, seed, p, n_a, n_b, 0, n_a, C);
  free(p);
  return 0;
}

/* array::matmul_gemm (array.hpp:85-95): C = AT^T B, k-ordered sums. */
void cmo_gemm(int64_t n_a, int64_t n_inner, int64_t n_b, double* C, const double* AT,
              const double* B) {
  for (int64_t i = 0; i < n_a; ++i)
    for (int64_t j = 0; j < n_b; ++j) {
      double s = 0.0;
      for (int64_t k = 0; k < n_inner; ++k) s += AT[k * n_a + i] * B[k * n_b + j];
      C[i * n_b + j] = s;
    }
}

/* The 64-bit seed used when the caller passes none: rng()() with the time
 * seed of rng.hpp:54-56, matmul_fft.hpp:30-32. */
uint64_t cmo_seed_from_time_millis(uint64_t millis) {
  uint64_t s[4];
  cmo_rng_seed(s, millis);
  return cmo_rng_next(s);
}
