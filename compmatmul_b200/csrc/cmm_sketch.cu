// Sketch kernels of the compressed product (the hot path).
//
// Reference algorithm (matmul_fft.hpp:25-129, matmul_fwht.hpp:25-114): for
// each inner index k and repetition t, count-sketch column k of A and row k
// of B into b buckets, transform both, multiply pointwise, accumulate over
// k, and finally inverse-transform the d accumulated spectra into p (d x b).
//
// B200 formulation:
//  * Hash codes are precomputed once per call, one u32 per (t, index):
//    bucket | (sign == +1) << 31 (k_hash_codes).  The reference re-hashes
//    per (k, t, i); the values are identical.
//  * A length-b transform does not fit one SM for b = 2^16 in FP64, so the
//    b frequencies are split into R = b / L slabs of L frequencies.  One CTA
//    owns one (repetition t, slab r) for a range of k and never exchanges
//    data with other CTAs:
//      FFT  (decimation in frequency): X[R m + r] = FFT_L(u_r)[m] with
//           u_r[n] = w_b^{n r} sum_q w_R^{q r} x[n + q L];
//      FWHT (Kronecker split): X[r L + m] = WHT_L(u_r)[m] with
//           u_r[n] = sum_q (-1)^{popc(q & r)} x[q L + n].
//    The CTA builds u_r directly by scattering each row element into
//    bucket n = h mod L with weight w_R^{(h div L) r} (or +-1): the count
//    sketch and the first transform stage are fused, and the n x b sketches
//    never reach HBM.
//  * FFT: the A side goes to the real part and the B side to the imaginary
//    part of one complex sequence z = alpha x + i beta y.  With Z = FFT(z),
//    X Y = (Z[f]^2 - conj(Z[-f])^2) / (4 i) (alpha beta = 1), so each CTA
//    only accumulates Q[f] += Z[f]^2 for its own frequencies; the pairing of
//    f with -f happens once, after the k loop (k_fft_combine).  alpha/beta
//    are per-k powers of two that balance the two halves (k_row_scale), so
//    the combination loses no precision when A and B rows differ in scale.
//  * FWHT: x and y stay separate real sequences; P[f] += X[f] Y[f].
//  * Per-CTA accumulators live in registers; partials of the G k-groups are
//    reduced in FP64 by the finalize kernels, which also run the inverse as
//    a two-pass (L then R) transform in global memory.
#include <cstdio>

#include "cmm_internal.h"

namespace cmm {

constexpr int kThreads = 512;
constexpr int kFftCap = 4096;                  // complex FP64 in the CTA buffer
constexpr int kFftQPT = kFftCap / kThreads;    // accumulator entries per thread
constexpr int kWhtCap = 8192;                  // real FP64 per buffer (x and y)
constexpr int kWhtQPT = kWhtCap / kThreads;
constexpr int kSkipRow = -0x7fffffff;          // row scale sentinel: A or B row is zero

// ----------------------------------------------------------------- helpers

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// bit reversal of the low `lg` bits (lg >= 1)
__device__ __forceinline__ uint32_t brev_bits(uint32_t x, int lg) { return __brev(x) >> (32 - lg); }

// exact 2^e for |e| <= 1000
__device__ __forceinline__ double exp2i(int e) {
  return __longlong_as_double((long long)(1023 + e) << 52);
}

// -------------------------------------------------------------- hash codes
// code = bucket | (sign == +1) << 31 for one function pair (H bucket
// function, S sign function) of family KIND; hashing.hpp:91-97, 163-169,
// 298-314.  Keys are u32 (the reference's key_t).
template <int KIND>
__device__ __forceinline__ uint32_t hash_code(const void* H, const void* S, int t, int log2b,
                                              uint32_t key) {
  uint32_t bucket, bit;
  if (KIND == MS) {
    const uint64_t a = reinterpret_cast<const uint64_t*>(H)[t];
    const uint64_t as = reinterpret_cast<const uint64_t*>(S)[t];
    bucket = (uint32_t)((a * (uint64_t)key) >> (64 - log2b));
    bit = (uint32_t)((as * (uint64_t)key) >> 63);
  } else if (KIND == MAS) {
    const uint64_t* ab = reinterpret_cast<const uint64_t*>(H) + 2 * t;
    const uint64_t* sb = reinterpret_cast<const uint64_t*>(S) + 2 * t;
    bucket = (uint32_t)((ab[0] * (uint64_t)key + ab[1]) >> (64 - log2b));
    bit = (uint32_t)((sb[0] * (uint64_t)key + sb[1]) >> 63);
  } else if (KIND == TAB8) {
    const uint32_t* T = reinterpret_cast<const uint32_t*>(H) + (size_t)t * 1024;
    const uint32_t* U = reinterpret_cast<const uint32_t*>(S) + (size_t)t * 1024;
    const uint32_t k0 = key & 0xffu, k1 = (key >> 8) & 0xffu, k2 = (key >> 16) & 0xffu, k3 = key >> 24;
    const uint32_t h = __ldg(T + k0) ^ __ldg(T + 256 + k1) ^ __ldg(T + 512 + k2) ^ __ldg(T + 768 + k3);
    const uint32_t g = __ldg(U + k0) ^ __ldg(U + 256 + k1) ^ __ldg(U + 512 + k2) ^ __ldg(U + 768 + k3);
    bucket = h >> (32 - log2b);
    bit = g >> 31;
  } else {
    const uint32_t* T = reinterpret_cast<const uint32_t*>(H) + (size_t)t * 131072;
    const uint32_t* U = reinterpret_cast<const uint32_t*>(S) + (size_t)t * 131072;
    const uint32_t h = __ldg(T + (key & 0xffffu)) ^ __ldg(T + 65536 + (key >> 16));
    const uint32_t g = __ldg(U + (key & 0xffffu)) ^ __ldg(U + 65536 + (key >> 16));
    bucket = h >> (32 - log2b);
    bit = g >> 31;
  }
  return bucket | (bit << 31);
}

template <int KIND>
__global__ void k_hash_codes(const void* H, const void* S, int d, int log2b, int64_t n,
                             const uint32_t* keys, uint32_t* codes) {
  const int t = blockIdx.y;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t key = keys ? keys[i] : (uint32_t)i;
    codes[(size_t)t * n + i] = hash_code<KIND>(H, S, t, log2b, key);
  }
}

void launch_hash_codes_keys(int kind, const void* dH, const void* dS, int d, int log2b, int64_t n,
                            const uint32_t* dKeys, uint32_t* dCodes, cudaStream_t s) {
  if (n <= 0 || d <= 0) return;
  const int threads = 256;
  int64_t blocks = (n + threads - 1) / threads;
  if (blocks > 4096) blocks = 4096;
  dim3 grid((unsigned)blocks, (unsigned)d);
  ProfScope prof("hash", s);
  count_launch();
  switch (kind) {
    case MS: k_hash_codes<MS><<<grid, threads, 0, s>>>(dH, dS, d, log2b, n, dKeys, dCodes); break;
    case MAS: k_hash_codes<MAS><<<grid, threads, 0, s>>>(dH, dS, d, log2b, n, dKeys, dCodes); break;
    case TAB8: k_hash_codes<TAB8><<<grid, threads, 0, s>>>(dH, dS, d, log2b, n, dKeys, dCodes); break;
    default: k_hash_codes<TAB16><<<grid, threads, 0, s>>>(dH, dS, d, log2b, n, dKeys, dCodes); break;
  }
  CMM_CUDA(cudaGetLastError());
}

void launch_hash_codes(int kind, const void* dH, const void* dS, int d, int log2b, int64_t n,
                       uint32_t* dCodes, cudaStream_t s) {
  launch_hash_codes_keys(kind, dH, dS, d, log2b, n, nullptr, dCodes, s);
}

// Many independent code sets in one launch (batched products): block row y
// serves job y; codes[t * n + i] for keys 0..n-1, t < d.
__global__ void k_hash_codes_jobs(const HashJob* __restrict__ jobs) {
  const HashJob J = jobs[blockIdx.y];
  const int64_t total = J.n * (int64_t)J.d;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / J.n);
    const uint32_t key = (uint32_t)(e - (int64_t)t * J.n);
    uint32_t c;
    switch (J.kind) {
      case MS: c = hash_code<MS>(J.H, J.S, t, J.log2b, key); break;
      case MAS: c = hash_code<MAS>(J.H, J.S, t, J.log2b, key); break;
      case TAB8: c = hash_code<TAB8>(J.H, J.S, t, J.log2b, key); break;
      default: c = hash_code<TAB16>(J.H, J.S, t, J.log2b, key); break;
    }
    J.codes[e] = c;
  }
}

void launch_hash_codes_jobs(const HashJob* dJobs, int njobs, int64_t max_total, cudaStream_t s) {
  if (njobs <= 0 || max_total <= 0) return;
  const int threads = 256;
  int64_t blocks = (max_total + threads - 1) / threads;
  if (blocks > 1024) blocks = 1024;
  ProfScope prof("hash", s);
  count_launch();
  k_hash_codes_jobs<<<dim3((unsigned)blocks, (unsigned)njobs), threads, 0, s>>>(dJobs);
  CMM_CUDA(cudaGetLastError());
}

// --------------------------------------------------------------- row scale
// e_k = round-to-zero((expo(max|AT[k,:]|) - expo(max|B[k,:]|)) / 2); the FFT
// kernel scales the A row by 2^-e_k and the B row by 2^e_k (exact).
__device__ __forceinline__ int expo_of(double m) {
  const long long bits = __double_as_longlong(m);
  return (int)((bits >> 52) & 0x7ff) - 1023;
}

__global__ void k_row_scale(const double* AT, const double* B, int64_t n_a, int64_t n_b,
                            int* scale_exp) {
  const int64_t k = blockIdx.x;
  const double* ra = AT + k * n_a;
  const double* rb = B + k * n_b;
  double ma = 0.0, mb = 0.0;
  for (int64_t i = threadIdx.x; i < n_a; i += blockDim.x) ma = fmax(ma, fabs(__ldg(ra + i)));
  for (int64_t j = threadIdx.x; j < n_b; j += blockDim.x) mb = fmax(mb, fabs(__ldg(rb + j)));
  for (int o = 16; o > 0; o >>= 1) {
    ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
    mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
  }
  __shared__ double sa[32], sb[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sa[w] = ma; sb[w] = mb; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) { ma = fmax(ma, sa[i]); mb = fmax(mb, sb[i]); }
    int e;
    if (!(ma > 0.0) || !(mb > 0.0)) {
      // a zero row contributes nothing; NaN rows keep e = 0 so NaN propagates
      e = (ma == 0.0 || mb == 0.0) ? kSkipRow : 0;
    } else {
      e = (expo_of(ma) - expo_of(mb)) / 2;
      e = e > 400 ? 400 : (e < -400 ? -400 : e);
    }
    scale_exp[k] = e;
  }
}

void launch_row_scale(const double* dAT, const double* dB, int64_t n_a, int64_t n_inner,
                      int64_t n_b, int* dScaleExp, cudaStream_t s) {
  if (n_inner <= 0) return;
  ProfScope prof("scale", s);
  count_launch();
  k_row_scale<<<(unsigned)n_inner, 256, 0, s>>>(dAT, dB, n_a, n_b, dScaleExp);
  CMM_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------- sketch args
struct SketchArgs {
  const double* AT;
  const double* B;
  const uint32_t* codesA;
  const uint32_t* codesB;
  const int* scale_exp;
  const double2* tw;
  void* partial;
  int64_t n_a, n_inner, n_b;
  int d, log2b, logL, logR, KB, G;
};

__device__ __forceinline__ void k_range(const SketchArgs& a, int g, int64_t& kb, int64_t& ke) {
  const int64_t per = (a.n_inner + a.G - 1) / a.G;
  kb = (int64_t)g * per;
  ke = kb + per < a.n_inner ? kb + per : a.n_inner;
}

// ----------------------------------------------------------- FFT variant
// grid (R, d, G); block kThreads; dynamic smem kFftCap * 16 bytes.
__global__ void __launch_bounds__(kThreads, 2) k_sketch_fft(SketchArgs a) {
  extern __shared__ double2 buf[];
  const int tid = threadIdx.x;
  const int r = blockIdx.x, t = blockIdx.y, g = blockIdx.z;
  const int logL = a.logL, L = 1 << logL, R = 1 << a.logR;
  const int nbuf = a.KB << logL;
  const uint32_t* cA = a.codesA + (size_t)t * a.n_a;
  const uint32_t* cB = a.codesB + (size_t)t * a.n_b;
  int64_t k_begin, k_end;
  k_range(a, g, k_begin, k_end);

  double2 q[kFftQPT];
#pragma unroll
  for (int j = 0; j < kFftQPT; ++j) q[j] = make_double2(0.0, 0.0);

  for (int64_t k0 = k_begin; k0 < k_end; k0 += a.KB) {
    for (int e = tid; e < nbuf; e += kThreads) buf[e] = make_double2(0.0, 0.0);
    __syncthreads();
    // --- fused count sketch + first transform stage (scatter)
    for (int kb = 0; kb < a.KB; ++kb) {
      const int64_t k = k0 + kb;
      if (k >= k_end) break;
      const int se = __ldg(a.scale_exp + k);
      if (se == kSkipRow) continue;
      const double alpha = exp2i(-se), beta = exp2i(se);
      const double* ra = a.AT + (size_t)k * a.n_a;
      const double* rb = a.B + (size_t)k * a.n_b;
      double2* seq = buf + (kb << logL);
      for (int64_t i = tid; i < a.n_a; i += kThreads) {
        const uint32_t c = __ldg(cA + i);
        double v = __ldg(ra + i) * alpha;
        if (!(c >> 31)) v = -v;
        const uint32_t h = c & 0x7fffffffu;
        double2* dst = seq + brev_bits(h & (uint32_t)(L - 1), logL);
        if (R == 1) {
          atomicAdd(&dst->x, v);
        } else {
          const double2 w = __ldg(a.tw + (((h >> logL) * (uint32_t)r & (uint32_t)(R - 1)) << logL));
          atomicAdd(&dst->x, v * w.x);
          atomicAdd(&dst->y, v * w.y);
        }
      }
      for (int64_t j = tid; j < a.n_b; j += kThreads) {
        const uint32_t c = __ldg(cB + j);
        double v = __ldg(rb + j) * beta;
        if (!(c >> 31)) v = -v;
        const uint32_t h = c & 0x7fffffffu;
        double2* dst = seq + brev_bits(h & (uint32_t)(L - 1), logL);
        if (R == 1) {
          atomicAdd(&dst->y, v);
        } else {
          const double2 w = __ldg(a.tw + (((h >> logL) * (uint32_t)r & (uint32_t)(R - 1)) << logL));
          atomicAdd(&dst->x, -v * w.y);
          atomicAdd(&dst->y, v * w.x);
        }
      }
    }
    __syncthreads();
    // --- twiddle w_b^{n r} (n = natural index of the bit-reversed slot)
    if (r != 0) {
      for (int e = tid; e < nbuf; e += kThreads) {
        const uint32_t n = brev_bits((uint32_t)(e & (L - 1)), logL);
        buf[e] = cmul(buf[e], __ldg(a.tw + n * (uint32_t)r));
      }
      __syncthreads();
    }
    // --- radix-2 DIT stages, bit-reversed in, natural order out
    for (int s = 0; s < logL; ++s) {
      const int half = 1 << s;
      for (int p = tid; p < (nbuf >> 1); p += kThreads) {
        const int base = (p >> (logL - 1)) << logL;
        const int jj = p & ((L >> 1) - 1);
        const int kk = jj & (half - 1);
        const int ia = base + ((jj >> s) << (s + 1)) + kk;
        const int ic = ia + half;
        const double2 w = __ldg(a.tw + ((uint32_t)kk << (a.log2b - s - 1)));
        const double2 u = buf[ia];
        const double2 v = cmul(buf[ic], w);
        buf[ia] = cadd(u, v);
        buf[ic] = csub(u, v);
      }
      __syncthreads();
    }
    // --- Q[m] += Z[m]^2 over the KB sequences
#pragma unroll
    for (int j = 0; j < kFftQPT; ++j) {
      const int m = tid + j * kThreads;
      if (m < L) {
        double2 acc = q[j];
        for (int kb = 0; kb < a.KB; ++kb) {
          const double2 z = buf[(kb << logL) + m];
          acc.x = fma(z.x, z.x, fma(-z.y, z.y, acc.x));
          acc.y = fma(2.0 * z.x, z.y, acc.y);
        }
        q[j] = acc;
      }
    }
    __syncthreads();
  }
  double2* out = reinterpret_cast<double2*>(a.partial) +
                 (((size_t)g * a.d + t) * (size_t)R + r) * (size_t)L;
#pragma unroll
  for (int j = 0; j < kFftQPT; ++j) {
    const int m = tid + j * kThreads;
    if (m < L) out[m] = q[j];
  }
}

// ---------------------------------------------------------- FWHT variant
// grid (R, d, G); dynamic smem 2 * kWhtCap * 8 bytes.
__global__ void __launch_bounds__(kThreads, 1) k_sketch_fwht(SketchArgs a) {
  extern __shared__ double wbuf[];
  double* xs = wbuf;
  double* ys = wbuf + kWhtCap;
  const int tid = threadIdx.x;
  const int r = blockIdx.x, t = blockIdx.y, g = blockIdx.z;
  const int logL = a.logL, L = 1 << logL;
  const int nbuf = a.KB << logL;
  const uint32_t* cA = a.codesA + (size_t)t * a.n_a;
  const uint32_t* cB = a.codesB + (size_t)t * a.n_b;
  int64_t k_begin, k_end;
  k_range(a, g, k_begin, k_end);

  double acc[kWhtQPT];
#pragma unroll
  for (int j = 0; j < kWhtQPT; ++j) acc[j] = 0.0;

  for (int64_t k0 = k_begin; k0 < k_end; k0 += a.KB) {
    for (int e = tid; e < nbuf; e += kThreads) { xs[e] = 0.0; ys[e] = 0.0; }
    __syncthreads();
    for (int kb = 0; kb < a.KB; ++kb) {
      const int64_t k = k0 + kb;
      if (k >= k_end) break;
      const double* ra = a.AT + (size_t)k * a.n_a;
      const double* rb = a.B + (size_t)k * a.n_b;
      double* sx = xs + (kb << logL);
      double* sy = ys + (kb << logL);
      for (int64_t i = tid; i < a.n_a; i += kThreads) {
        const uint32_t c = __ldg(cA + i);
        const uint32_t h = c & 0x7fffffffu;
        double v = __ldg(ra + i);
        // sign(+-1) * (-1)^{popc(q & r)}: negate when the parity bit differs
        const uint32_t neg = ((c >> 31) ^ 1u) ^ (__popc((h >> logL) & (uint32_t)r) & 1u);
        if (neg) v = -v;
        atomicAdd(sx + (h & (uint32_t)(L - 1)), v);
      }
      for (int64_t j = tid; j < a.n_b; j += kThreads) {
        const uint32_t c = __ldg(cB + j);
        const uint32_t h = c & 0x7fffffffu;
        double v = __ldg(rb + j);
        const uint32_t neg = ((c >> 31) ^ 1u) ^ (__popc((h >> logL) & (uint32_t)r) & 1u);
        if (neg) v = -v;
        atomicAdd(sy + (h & (uint32_t)(L - 1)), v);
      }
    }
    __syncthreads();
    for (int s = 0; s < logL; ++s) {
      const int half = 1 << s;
      for (int p = tid; p < (nbuf >> 1); p += kThreads) {
        const int base = (p >> (logL - 1)) << logL;
        const int jj = p & ((L >> 1) - 1);
        const int ia = base + ((jj >> s) << (s + 1)) + (jj & (half - 1));
        const int ic = ia + half;
        const double u = xs[ia], v = xs[ic];
        xs[ia] = u + v;
        xs[ic] = u - v;
        const double uy = ys[ia], vy = ys[ic];
        ys[ia] = uy + vy;
        ys[ic] = uy - vy;
      }
      __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < kWhtQPT; ++j) {
      const int m = tid + j * kThreads;
      if (m < L) {
        double s_ = acc[j];
        for (int kb = 0; kb < a.KB; ++kb) s_ = fma(xs[(kb << logL) + m], ys[(kb << logL) + m], s_);
        acc[j] = s_;
      }
    }
    __syncthreads();
  }
  double* out = reinterpret_cast<double*>(a.partial) +
                (((size_t)g * a.d + t) * (size_t)(1 << a.logR) + r) * (size_t)L;
#pragma unroll
  for (int j = 0; j < kWhtQPT; ++j) {
    const int m = tid + j * kThreads;
    if (m < L) out[m] = acc[j];
  }
}

// ------------------------------------------------------------------ plan
SketchPlan plan_sketch(int variant, int64_t n_a, int64_t n_inner, int64_t n_b, int d, int b,
                       int sms) {
  SketchPlan P{};
  P.variant = variant;
  P.d = d;
  P.b = b;
  P.log2b = 0;
  while ((1 << P.log2b) < b) ++P.log2b;
  const int lmax = variant == kVariantFFT ? kFftLmaxLog : kFwhtLmaxLog;
  P.logL = P.log2b < lmax ? P.log2b : lmax;
  P.L = 1 << P.logL;
  P.logR = P.log2b - P.logL;
  P.R = 1 << P.logR;
  const int cap = variant == kVariantFFT ? kFftCap : kWhtCap;
  P.KB = cap / P.L;
  P.n_a = n_a;
  P.n_inner = n_inner;
  P.n_b = n_b;
  const int per_sm = variant == kVariantFFT ? 2 : 1;
  const int64_t slots = (int64_t)sms * per_sm;
  const int64_t ctas_per_group = (int64_t)P.R * d;
  int64_t G = (slots + ctas_per_group - 1) / ctas_per_group;
  if (G < 1) G = 1;
  const int64_t max_groups = (n_inner + P.KB - 1) / P.KB;
  if (G > max_groups) G = max_groups;
  if (G < 1) G = 1;
  if (G > 65535) G = 65535;
  P.G = (int)G;
  return P;
}

void launch_sketch_accumulate(const SketchPlan& P, const double* dAT, const double* dB,
                              const uint32_t* dCodesA, const uint32_t* dCodesB,
                              const int* dScaleExp, const double2* dTw, void* dPartial,
                              cudaStream_t s) {
  SketchArgs a;
  a.AT = dAT;
  a.B = dB;
  a.codesA = dCodesA;
  a.codesB = dCodesB;
  a.scale_exp = dScaleExp;
  a.tw = dTw;
  a.partial = dPartial;
  a.n_a = P.n_a;
  a.n_inner = P.n_inner;
  a.n_b = P.n_b;
  a.d = P.d;
  a.log2b = P.log2b;
  a.logL = P.logL;
  a.logR = P.logR;
  a.KB = P.KB;
  a.G = P.G;
  dim3 grid((unsigned)P.R, (unsigned)P.d, (unsigned)P.G);
  if (P.variant == kVariantFFT) {
    const int smem = kFftCap * (int)sizeof(double2);
    CMM_CUDA(cudaFuncSetAttribute(k_sketch_fft, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ProfScope prof("sketch", s);
    count_launch();
    k_sketch_fft<<<grid, kThreads, smem, s>>>(a);
  } else {
    const int smem = 2 * kWhtCap * (int)sizeof(double);
    CMM_CUDA(cudaFuncSetAttribute(k_sketch_fwht, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ProfScope prof("sketch", s);
    count_launch();
    k_sketch_fwht<<<grid, kThreads, smem, s>>>(a);
  }
  CMM_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------- finalize
// FFT: P[f] = (Q[f] - conj(Q[-f])) / (4i), Q = sum over k groups; layout
// [t][r][m] with f = R m + r.
__global__ void k_fft_combine(const double2* partial, int G, int d, int logL, int logR,
                              double2* Pout) {
  const int L = 1 << logL, R = 1 << logR;
  const int64_t b = (int64_t)L * R;
  const int64_t total = (int64_t)d * b;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(idx / b);
    const int64_t rem = idx - (int64_t)t * b;
    const int r = (int)(rem >> logL);
    const int m = (int)(rem & (L - 1));
    const int rn = (R - r) & (R - 1);
    const int mn = r == 0 ? ((L - m) & (L - 1)) : (L - m - 1);
    double2 Q = make_double2(0.0, 0.0), Qn = make_double2(0.0, 0.0);
    for (int g = 0; g < G; ++g) {
      const double2* base = partial + ((size_t)g * d + t) * (size_t)b;
      const double2 u = base[((size_t)r << logL) + m];
      const double2 v = base[((size_t)rn << logL) + mn];
      Q.x += u.x; Q.y += u.y;
      Qn.x += v.x; Qn.y += v.y;
    }
    const double dx = Q.x - Qn.x, dy = Q.y + Qn.y;
    Pout[idx] = make_double2(0.25 * dy, -0.25 * dx);
  }
}

// FFT, partials in natural order [g][t][f]: P[f] = (Q[f] - conj(Q[-f]))/(4i),
// written in the [t][r][m] (f = R m + r) layout the inverse passes read.
__global__ void k_fft_combine_natural(const double2* partial, int G, int d, int log2b, int logL,
                                      double2* Pout) {
  const int64_t b = (int64_t)1 << log2b;
  const int logR = log2b - logL;
  const int64_t total = (int64_t)d * b;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(idx >> log2b);
    const int64_t f = idx & (b - 1);
    const int64_t fn = (b - f) & (b - 1);
    double2 Q = make_double2(0.0, 0.0), Qn = make_double2(0.0, 0.0);
    for (int g = 0; g < G; ++g) {
      const double2* base = partial + ((size_t)g * d + t) * (size_t)b;
      const double2 u = base[f], v = base[fn];
      Q.x += u.x; Q.y += u.y;
      Qn.x += v.x; Qn.y += v.y;
    }
    const double dx = Q.x - Qn.x, dy = Q.y + Qn.y;
    const int64_t r = f & (((int64_t)1 << logR) - 1), m = f >> logR;
    Pout[(size_t)t * b + ((size_t)r << logL) + m] = make_double2(0.25 * dy, -0.25 * dx);
  }
}

// FWHT: sum of the k-group partials.
__global__ void k_sum_partials(const double* partial, int G, int64_t n, double* out) {
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    double s_ = 0.0;
    for (int g = 0; g < G; ++g) s_ += partial[(size_t)g * n + idx];
    out[idx] = s_;
  }
}

// Batched inverse transforms in shared memory.  Sequence s = (s1, s2) with
// s1 = s / inner, s2 = s % inner; element e of sequence s is read from
// in[s1*is1 + s2*is2 + e*ie] and written to out[s1*os1 + s2*os2 + e*oe].
struct BatchArgs {
  const void* in;
  void* out;
  int logM;
  int64_t nseq, inner;
  int64_t is1, is2, ie, os1, os2, oe;
  const double2* tw;
  int log2b;
  int post;      // FFT: 1 = multiply by w_b^{-s2*e} (complex out); 2 = real part * scale out
  double scale;  // WHT: applied to the output
};

__device__ __forceinline__ void seq_addr(const BatchArgs& a, int64_t s, int64_t& ib, int64_t& ob) {
  const int64_t s1 = s / a.inner, s2 = s - s1 * a.inner;
  ib = s1 * a.is1 + s2 * a.is2;
  ob = s1 * a.os1 + s2 * a.os2;
}

constexpr int kBatchThreads = 256;
constexpr int kBatchFftCap = 8192;  // complex FP64 per CTA (slabs up to L = 8192)

// inverse complex DFT (sign +1), unnormalised
__global__ void __launch_bounds__(kBatchThreads) k_batch_ifft(BatchArgs a) {
  extern __shared__ double2 sb[];
  const int M = 1 << a.logM;
  const int spc = kBatchFftCap >> a.logM;  // sequences per CTA
  const int64_t s0 = (int64_t)blockIdx.x * spc;
  const double2* in = reinterpret_cast<const double2*>(a.in);
  for (int e = threadIdx.x; e < (spc << a.logM); e += kBatchThreads) {
    const int sl = e >> a.logM, el = e & (M - 1);
    const int64_t s = s0 + sl;
    double2 v = make_double2(0.0, 0.0);
    if (s < a.nseq) {
      int64_t ib, ob;
      seq_addr(a, s, ib, ob);
      v = in[ib + el * a.ie];
    }
    const int pos = a.logM ? (int)brev_bits((uint32_t)el, a.logM) : 0;
    sb[(sl << a.logM) + pos] = v;
  }
  __syncthreads();
  for (int st = 0; st < a.logM; ++st) {
    const int half = 1 << st;
    for (int p = threadIdx.x; p < ((spc << a.logM) >> 1); p += kBatchThreads) {
      const int base = (p >> (a.logM - 1)) << a.logM;
      const int jj = p & ((M >> 1) - 1);
      const int kk = jj & (half - 1);
      const int ia = base + ((jj >> st) << (st + 1)) + kk;
      const int ic = ia + half;
      const double2 w = a.tw[(uint32_t)kk << (a.log2b - st - 1)];
      const double2 u = sb[ia];
      const double2 v = cmulc(sb[ic], w);
      sb[ia] = cadd(u, v);
      sb[ic] = csub(u, v);
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < (spc << a.logM); e += kBatchThreads) {
    const int sl = e >> a.logM, el = e & (M - 1);
    const int64_t s = s0 + sl;
    if (s >= a.nseq) continue;
    int64_t ib, ob;
    seq_addr(a, s, ib, ob);
    double2 z = sb[e];
    if (a.post == 1) {
      const int64_t s2 = s % a.inner;
      z = cmulc(z, a.tw[(uint64_t)s2 * (uint64_t)el]);
      reinterpret_cast<double2*>(a.out)[ob + el * a.oe] = z;
    } else {
      reinterpret_cast<double*>(a.out)[ob + el * a.oe] = z.x * a.scale;
    }
  }
}

// unnormalised natural-order WHT of real sequences, output * scale
__global__ void __launch_bounds__(kBatchThreads) k_batch_wht(BatchArgs a) {
  extern __shared__ double sw[];
  const int M = 1 << a.logM;
  const int spc = kWhtCap >> a.logM;
  const int64_t s0 = (int64_t)blockIdx.x * spc;
  const double* in = reinterpret_cast<const double*>(a.in);
  for (int e = threadIdx.x; e < (spc << a.logM); e += kBatchThreads) {
    const int sl = e >> a.logM, el = e & (M - 1);
    const int64_t s = s0 + sl;
    double v = 0.0;
    if (s < a.nseq) {
      int64_t ib, ob;
      seq_addr(a, s, ib, ob);
      v = in[ib + el * a.ie];
    }
    sw[e] = v;
  }
  __syncthreads();
  for (int st = 0; st < a.logM; ++st) {
    const int half = 1 << st;
    for (int p = threadIdx.x; p < ((spc << a.logM) >> 1); p += kBatchThreads) {
      const int base = (p >> (a.logM - 1)) << a.logM;
      const int jj = p & ((M >> 1) - 1);
      const int ia = base + ((jj >> st) << (st + 1)) + (jj & (half - 1));
      const int ic = ia + half;
      const double u = sw[ia], v = sw[ic];
      sw[ia] = u + v;
      sw[ic] = u - v;
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < (spc << a.logM); e += kBatchThreads) {
    const int sl = e >> a.logM, el = e & (M - 1);
    const int64_t s = s0 + sl;
    if (s >= a.nseq) continue;
    int64_t ib, ob;
    seq_addr(a, s, ib, ob);
    reinterpret_cast<double*>(a.out)[ob + el * a.oe] = sw[e] * a.scale;
  }
}

static void run_batch(bool fft, BatchArgs a, cudaStream_t s) {
  const int cap = fft ? kBatchFftCap : kWhtCap;
  const int spc = cap >> a.logM;
  const int64_t blocks = (a.nseq + spc - 1) / spc;
  const int smem = fft ? kBatchFftCap * (int)sizeof(double2) : kWhtCap * (int)sizeof(double);
  count_launch();
  if (fft) {
    CMM_CUDA(cudaFuncSetAttribute(k_batch_ifft, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_batch_ifft<<<(unsigned)blocks, kBatchThreads, smem, s>>>(a);
  } else {
    CMM_CUDA(cudaFuncSetAttribute(k_batch_wht, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_batch_wht<<<(unsigned)blocks, kBatchThreads, smem, s>>>(a);
  }
  CMM_CUDA(cudaGetLastError());
}

// dWork holds 2 * d * b * 16 bytes.
void launch_finalize(const SketchPlan& P, const void* dPartial, const double2* dTw, void* dWork,
                     double* dP, cudaStream_t s) {
  const int64_t db = (int64_t)P.d * P.b;
  int64_t blocks = (db + 255) / 256;
  if (blocks > 8192) blocks = 8192;
  const double inv_b = 1.0 / (double)P.b;
  ProfScope prof("finalize", s);
  count_launch(3);
  if (P.variant == kVariantFFT) {
    double2* w1 = reinterpret_cast<double2*>(dWork);
    double2* w2 = w1 + db;
    k_fft_combine<<<(unsigned)blocks, 256, 0, s>>>(reinterpret_cast<const double2*>(dPartial), P.G,
                                                   P.d, P.logL, P.logR, w1);
    CMM_CUDA(cudaGetLastError());
    // step 1: v_r[n] = sum_m w_L^{-mn} P[t][r][m], times w_b^{-rn}
    BatchArgs a{};
    a.in = w1; a.out = w2; a.logM = P.logL;
    a.nseq = (int64_t)P.d * P.R; a.inner = P.R;
    a.is1 = P.b; a.is2 = P.L; a.ie = 1;
    a.os1 = P.b; a.os2 = P.L; a.oe = 1;
    a.tw = dTw; a.log2b = P.log2b; a.post = 1; a.scale = 1.0;
    run_batch(true, a, s);
    // step 2: p[t][n + qL] = (1/b) Re sum_r w_R^{-rq} v_r[n]
    BatchArgs c{};
    c.in = w2; c.out = dP; c.logM = P.logR;
    c.nseq = (int64_t)P.d * P.L; c.inner = P.L;
    c.is1 = P.b; c.is2 = 1; c.ie = P.L;
    c.os1 = P.b; c.os2 = 1; c.oe = P.L;
    c.tw = dTw; c.log2b = P.log2b; c.post = 2; c.scale = inv_b;
    run_batch(true, c, s);
  } else {
    double* w1 = reinterpret_cast<double*>(dWork);
    double* w2 = w1 + db;
    k_sum_partials<<<(unsigned)blocks, 256, 0, s>>>(reinterpret_cast<const double*>(dPartial), P.G,
                                                    db, w1);
    CMM_CUDA(cudaGetLastError());
    BatchArgs a{};
    a.in = w1; a.out = w2; a.logM = P.logL;
    a.nseq = (int64_t)P.d * P.R; a.inner = P.R;
    a.is1 = P.b; a.is2 = P.L; a.ie = 1;
    a.os1 = P.b; a.os2 = P.L; a.oe = 1;
    a.tw = dTw; a.log2b = P.log2b; a.post = 0; a.scale = 1.0;
    run_batch(false, a, s);
    BatchArgs c{};
    c.in = w2; c.out = dP; c.logM = P.logR;
    c.nseq = (int64_t)P.d * P.L; c.inner = P.L;
    c.is1 = P.b; c.is2 = 1; c.ie = P.L;
    c.os1 = P.b; c.os2 = 1; c.oe = P.L;
    c.tw = dTw; c.log2b = P.log2b; c.post = 0; c.scale = inv_b;
    run_batch(false, c, s);
  }
}

void launch_finalize_natural(int variant, int d, int b, int G, const void* dPartial,
                             const double2* dTw, void* dWork, double* dP, cudaStream_t s) {
  SketchPlan P{};
  P.variant = variant;
  P.d = d;
  P.b = b;
  P.log2b = 0;
  while ((1 << P.log2b) < b) ++P.log2b;
  P.logL = P.log2b < 12 ? P.log2b : 12;
  P.L = 1 << P.logL;
  P.logR = P.log2b - P.logL;
  P.R = 1 << P.logR;
  P.G = G;
  if (variant != kVariantFFT) {
    // FWHT partials are already in natural order = the [t][r][m] layout
    launch_finalize(P, dPartial, dTw, dWork, dP, s);
    return;
  }
  const int64_t db = (int64_t)d * b;
  int64_t blocks = (db + 255) / 256;
  if (blocks > 8192) blocks = 8192;
  ProfScope prof("finalize", s);
  count_launch(3);
  double2* w1 = reinterpret_cast<double2*>(dWork);
  double2* w2 = w1 + db;
  k_fft_combine_natural<<<(unsigned)blocks, 256, 0, s>>>(reinterpret_cast<const double2*>(dPartial), G, d,
                                                         P.log2b, P.logL, w1);
  CMM_CUDA(cudaGetLastError());
  BatchArgs a{};
  a.in = w1; a.out = w2; a.logM = P.logL;
  a.nseq = (int64_t)P.d * P.R; a.inner = P.R;
  a.is1 = P.b; a.is2 = P.L; a.ie = 1;
  a.os1 = P.b; a.os2 = P.L; a.oe = 1;
  a.tw = dTw; a.log2b = P.log2b; a.post = 1; a.scale = 1.0;
  run_batch(true, a, s);
  BatchArgs c{};
  c.in = w2; c.out = dP; c.logM = P.logR;
  c.nseq = (int64_t)P.d * P.L; c.inner = P.L;
  c.is1 = P.b; c.is2 = 1; c.ie = P.L;
  c.os1 = P.b; c.os2 = 1; c.oe = P.L;
  c.tw = dTw; c.log2b = P.log2b; c.post = 2; c.scale = 1.0 / (double)P.b;
  run_batch(true, c, s);
}

}  // namespace cmm
