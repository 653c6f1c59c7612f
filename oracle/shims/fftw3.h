// Project-written stand-in for the subset of the FFTW3 API that the
// reference's transform.hpp uses (transform.hpp:28,42-48,59,70):
// fftw_plan_dft_r2c_1d / fftw_plan_dft_c2r_1d / fftw_execute /
// fftw_destroy_plan / fftw_malloc / fftw_free / FFTW_MEASURE.
// FFTW is not installed in this image.  This header lets the reference's
// own headers compile unchanged for the CPU oracle and baseline; it is test
// infrastructure, never part of the product.
//
// Semantics follow FFTW's documented r2c/c2r definitions: r2c computes
// X[f] = sum_h x[h] exp(-2 pi i f h / n) for f = 0..n/2 (unnormalised);
// c2r computes x[h] = sum_f X[f] exp(+2 pi i f h / n) over the Hermitian
// extension, unnormalised, ignoring Im X[0] and Im X[n/2].
// Algorithm: real length-n transform through one complex length-n/2
// radix-2 transform and the standard even/odd split.
#ifndef CMM_SHIM_FFTW3_H
#define CMM_SHIM_FFTW3_H

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

typedef double fftw_complex[2];

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

struct cmm_shim_fftw_plan {
  int n;          // real length
  int kind;       // 0 = r2c, 1 = c2r
  double* real;   // real buffer (in for r2c, out for c2r)
  fftw_complex* cplx;
  std::vector<std::complex<double>> tw_half;  // exp(-2 pi i k / (n/2)), k < n/4 .. n/2
  std::vector<std::complex<double>> tw_full;  // exp(-2 pi i f / n), f <= n/2
  std::vector<std::complex<double>> work;
  std::vector<int> rev;
};
typedef cmm_shim_fftw_plan* fftw_plan;

inline void* fftw_malloc(size_t n) {
  size_t bytes = (n + 63) / 64 * 64;
  return aligned_alloc(64, bytes ? bytes : 64);
}
inline void fftw_free(void* p) { free(p); }

namespace cmm_shim_detail {
inline void setup(cmm_shim_fftw_plan* p) {
  const int n = p->n;
  const int m = n / 2;
  const long double two_pi = 6.283185307179586476925286766559005768L;
  p->tw_full.resize(m + 1);
  for (int f = 0; f <= m; ++f) {
    long double a = -two_pi * f / n;
    p->tw_full[f] = std::complex<double>((double)cosl(a), (double)sinl(a));
  }
  if (m >= 1) {
    p->tw_half.resize(m > 1 ? m / 2 : 1);
    for (int k = 0; k < (int)p->tw_half.size(); ++k) {
      long double a = -two_pi * k / m;
      p->tw_half[k] = std::complex<double>((double)cosl(a), (double)sinl(a));
    }
    p->rev.resize(m);
    int lg = 0;
    while ((1 << lg) < m) ++lg;
    for (int i = 0; i < m; ++i) {
      int r = 0;
      for (int bit = 0; bit < lg; ++bit)
        if (i & (1 << bit)) r |= 1 << (lg - 1 - bit);
      p->rev[i] = r;
    }
    p->work.resize(m);
  }
}

// In-place complex DFT of length m (power of 2) on p->work; sign -1 forward.
inline void cfft(cmm_shim_fftw_plan* p, int sign) {
  const int m = p->n / 2;
  std::complex<double>* z = p->work.data();
  for (int i = 0; i < m; ++i)
    if (i < p->rev[i]) std::swap(z[i], z[p->rev[i]]);
  for (int len = 2; len <= m; len <<= 1) {
    const int half = len >> 1;
    const int step = m / len;
    for (int s = 0; s < m; s += len) {
      for (int k = 0; k < half; ++k) {
        std::complex<double> w = p->tw_half[k * step];
        if (sign > 0) w = std::conj(w);
        const std::complex<double> x = z[s + k + half] * w;
        z[s + k + half] = z[s + k] - x;
        z[s + k] += x;
      }
    }
  }
}
}  // namespace cmm_shim_detail

inline fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned) {
  cmm_shim_fftw_plan* p = new cmm_shim_fftw_plan();
  p->n = n; p->kind = 0; p->real = in; p->cplx = out;
  cmm_shim_detail::setup(p);
  return p;
}

inline fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex* in, double* out, unsigned) {
  cmm_shim_fftw_plan* p = new cmm_shim_fftw_plan();
  p->n = n; p->kind = 1; p->real = out; p->cplx = in;
  cmm_shim_detail::setup(p);
  return p;
}

inline void fftw_destroy_plan(fftw_plan p) { delete p; }

inline void fftw_execute(const fftw_plan p) {
  const int n = p->n;
  const int m = n / 2;
  typedef std::complex<double> cd;
  if (n == 1) {
    if (p->kind == 0) { p->cplx[0][0] = p->real[0]; p->cplx[0][1] = 0.0; }
    else p->real[0] = p->cplx[0][0];
    return;
  }
  if (p->kind == 0) {
    cd* z = p->work.data();
    for (int i = 0; i < m; ++i) z[i] = cd(p->real[2 * i], p->real[2 * i + 1]);
    cmm_shim_detail::cfft(p, -1);
    for (int f = 0; f <= m; ++f) {
      const cd a = z[f % m];
      const cd c = std::conj(z[(m - f) % m]);
      const cd E = 0.5 * (a + c);
      const cd O = cd(0.0, -0.5) * (a - c);
      const cd X = E + p->tw_full[f] * O;
      p->cplx[f][0] = X.real();
      p->cplx[f][1] = X.imag();
    }
  } else {
    cd* z = p->work.data();
    for (int f = 0; f < m; ++f) {
      cd a(p->cplx[f][0], f == 0 ? 0.0 : p->cplx[f][1]);
      const int g = m - f;
      cd c(p->cplx[g][0], (g == 0 || g == m) ? 0.0 : p->cplx[g][1]);
      c = std::conj(c);
      const cd E2 = a + c;
      const cd O2 = (a - c) * std::conj(p->tw_full[f]);
      z[f] = E2 + cd(0.0, 1.0) * O2;
    }
    cmm_shim_detail::cfft(p, +1);
    for (int i = 0; i < m; ++i) {
      p->real[2 * i] = z[i].real();
      p->real[2 * i + 1] = z[i].imag();
    }
  }
}

#endif  // CMM_SHIM_FFTW3_H
