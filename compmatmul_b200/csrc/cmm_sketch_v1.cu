// Sketch kernels v1: the hot path for b >= 4096 (FFT) / b >= 8192 (FWHT).
//
// Same decomposition as the v0 kernels (one CTA per (slab r, repetition t,
// k-group); the count sketch is fused with the first transform stage), but
// the rows arrive bucket-sorted and thread-interleaved (cmm_plan.cu):
//  * scatter: thread j owns a contiguous bucket range; it walks its slots
//    (coalesced loads, codes from shared memory), sums each run of equal
//    buckets in registers and stores each bucket once -- no atomics;
//  * transform: radix-8 (and radix-16) passes in registers on a padded
//    shared-memory layout (bank-conflict free for every pass);
//  * accumulation: the last pass leaves frequency m = tid + 512 e (FFT) or
//    m = g + 1024 e (FWHT) in the registers of its owner thread, which adds
//    Z^2 (or X*Y) into register accumulators without writing back.
#include "cmm_internal.h"

namespace cmm {

constexpr int kT = kPlanThreads;  // 512
constexpr int kSkip = -0x7fffffff;
constexpr int kBatch = 8;  // slots loaded ahead per thread in the scatter loops

// ---------------------------------------------------------------- FFT
constexpr int kFL = 4096, kFLog = 12;
constexpr int kFPhys = kFL + kFL / 8;  // padded: phys(p) = p + p / 8
__device__ __forceinline__ int fphys(int p) { return p + (p >> 3); }

// ---------------------------------------------------------------- WHT
constexpr int kWL = 8192, kWLog = 13;
constexpr int kWPhys = kWL + kWL / 16;  // padded: phys(p) = p + p / 16
__device__ __forceinline__ int wphys(int p) { return p + (p >> 4); }

struct V1Args {
  const double* matA;
  const double* matB;
  const void* codeA;
  const void* codeB;
  const uint32_t* countA;
  const uint32_t* countB;
  const int* scale_exp;
  const double2* tw;
  void* partial;
  int64_t SA, SB, kc, k0;
  int d, log2b, logR, G, accumulate, codes_in_smem;
};

__device__ __forceinline__ double2 c2(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return c2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 csq(double2 a) { return c2(fma(a.x, a.x, -a.y * a.y), 2.0 * a.x * a.y); }
__device__ __forceinline__ void bfly(double2& a, double2& b, double2 w) {
  const double2 t = cm(b, w);
  b = c2(a.x - t.x, a.y - t.y);
  a = c2(a.x + t.x, a.y + t.y);
}
__device__ __forceinline__ void bfly1(double2& a, double2& b) {  // twiddle 1
  const double2 t = b;
  b = c2(a.x - t.x, a.y - t.y);
  a = c2(a.x + t.x, a.y + t.y);
}

// three radix-2 DIT stages on points base + e*half (e < 8) in registers;
// W = w_{8 half}^{kk}.  Stage twiddles: W^4; W^2 w_4^{e mod 2}; W w_8^e.
__device__ __forceinline__ void r8_dit(double2 (&x)[8], double2 W) {
  const double h = 0.70710678118654752440;  // sqrt(2)/2
  const double2 W2 = csq(W), W4 = csq(W2);
  bfly(x[0], x[1], W4); bfly(x[2], x[3], W4); bfly(x[4], x[5], W4); bfly(x[6], x[7], W4);
  const double2 W2m = c2(W2.y, -W2.x);  // W2 * (-i)
  bfly(x[0], x[2], W2); bfly(x[4], x[6], W2); bfly(x[1], x[3], W2m); bfly(x[5], x[7], W2m);
  const double2 W1 = cm(W, c2(h, -h));   // W * w_8
  const double2 Wi = c2(W.y, -W.x);      // W * w_8^2 = W * (-i)
  const double2 W3 = cm(W, c2(-h, -h));  // W * w_8^3
  bfly(x[0], x[4], W); bfly(x[1], x[5], W1); bfly(x[2], x[6], Wi); bfly(x[3], x[7], W3);
}

__device__ __forceinline__ uint32_t brev12(uint32_t n) { return __brev(n) >> 20; }

template <typename CodeT>
__global__ void __launch_bounds__(kT, 1) k_sketch_fft_v1(V1Args a) {
  extern __shared__ __align__(16) unsigned char sm[];
  double2* buf = reinterpret_cast<double2*>(sm);
  double2* ptHi = buf + kFPhys;  // w_b^{64 x r}, x < 64
  double2* ptLo = ptHi + 64;     // w_b^{y r},    y < 64
  double2* tw1 = ptLo + 64;      // w_64^kk,   kk < 8
  double2* tw2 = tw1 + 8;        // w_512^kk,  kk < 64
  double2* tw3 = tw2 + 64;       // w_4096^kk, kk < 512
  double* wRx = reinterpret_cast<double*>(tw3 + 512);  // Re w_R^j, j < min(R, 256)
  double* wRy = wRx + 256;                              // Im w_R^j (separate: conflict-free)
  CodeT* cA = reinterpret_cast<CodeT*>(wRy + 256);
  CodeT* cB = cA + (a.codes_in_smem ? a.SA : 0);

  const int tid = threadIdx.x;
  const int r = blockIdx.x, t = blockIdx.y, g = blockIdx.z;
  const int R = 1 << a.logR;
  const double2* tw = a.tw;
  for (int e = tid; e < 64; e += kT) {
    ptHi[e] = tw[(uint32_t)(64 * e) * (uint32_t)r];
    ptLo[e] = tw[(uint32_t)e * (uint32_t)r];
    tw2[e] = tw[(uint32_t)e << (a.log2b - 9)];
  }
  for (int e = tid; e < 8; e += kT) tw1[e] = tw[(uint32_t)e << (a.log2b - 6)];
  for (int e = tid; e < 512; e += kT) tw3[e] = tw[(uint32_t)e << (a.log2b - 12)];
  for (int e = tid; e < (R < 256 ? R : 256); e += kT) {
    const double2 w = tw[(uint32_t)e << kFLog];
    wRx[e] = w.x;
    wRy[e] = w.y;
  }
  const CodeT* gA = reinterpret_cast<const CodeT*>(a.codeA) + (size_t)t * a.SA;
  const CodeT* gB = reinterpret_cast<const CodeT*>(a.codeB) + (size_t)t * a.SB;
  // shared codes carry (n, j) with j = (q r) mod R the slab weight index
  if (a.codes_in_smem) {
    for (int64_t e = tid; e < a.SA; e += kT) {
      const uint32_t h = gA[e];
      cA[e] = (CodeT)((h & (kFL - 1)) | ((((h >> kFLog) * (uint32_t)r) & (uint32_t)(R - 1)) << kFLog));
    }
    for (int64_t e = tid; e < a.SB; e += kT) {
      const uint32_t h = gB[e];
      cB[e] = (CodeT)((h & (kFL - 1)) | ((((h >> kFLog) * (uint32_t)r) & (uint32_t)(R - 1)) << kFLog));
    }
  }
  const bool premixed = a.codes_in_smem != 0;
  const CodeT* codesA = a.codes_in_smem ? cA : gA;
  const CodeT* codesB = a.codes_in_smem ? cB : gB;
  const int cntA = (int)a.countA[(size_t)t * kT + tid];
  const int cntB = (int)a.countB[(size_t)t * kT + tid];

  double2* part = reinterpret_cast<double2*>(a.partial) + (((size_t)g * a.d + t) * (size_t)R + r) * kFL;
  double2 q[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) q[e] = a.accumulate ? part[tid + 512 * e] : c2(0.0, 0.0);

  const int64_t per = (a.kc + a.G - 1) / a.G;
  const int64_t kb = (int64_t)g * per;
  const int64_t ke = kb + per < a.kc ? kb + per : a.kc;
  __syncthreads();

  for (int64_t kk = kb; kk < ke; ++kk) {
    const int se = __ldg(a.scale_exp + a.k0 + kk);
    if (se == kSkip) continue;  // uniform across the CTA
    for (int e = tid; e < kFPhys; e += kT) buf[e] = c2(0.0, 0.0);
    const double alpha = __longlong_as_double((long long)(1023 - se) << 52);
    const double beta = __longlong_as_double((long long)(1023 + se) << 52);
    __syncthreads();
    // ---- A side: real part, weights w_R^{q r}; one owner per bucket
    {
      const double* row = a.matA + ((size_t)t * a.kc + kk) * a.SA;
      uint32_t cur = 0xffffffffu;
      double2 acc = c2(0.0, 0.0);
      for (int s0 = 0; s0 < cntA; s0 += kBatch) {
        // issue the batch's loads first (independent), then consume
        double vv[kBatch];
        uint32_t hh[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          const bool ok = s0 + u < cntA;
          const int64_t e = (int64_t)(s0 + u) * kT + tid;
          vv[u] = ok ? __ldg(row + e) : 0.0;
          hh[u] = ok ? (uint32_t)codesA[e] : 0xffffffffu;
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          if (hh[u] == 0xffffffffu) break;
          const double v = vv[u];
          const uint32_t h = hh[u];
          const uint32_t n = h & (kFL - 1);
          double wx = 1.0, wy = 0.0;
          if (R > 1) {
            const uint32_t j = premixed ? (h >> kFLog) : (((h >> kFLog) * (uint32_t)r) & (uint32_t)(R - 1));
            if (j < 256) { wx = wRx[j]; wy = wRy[j]; }
            else { const double2 w = __ldg(tw + (j << kFLog)); wx = w.x; wy = w.y; }
          }
          if (n != cur) {
            if (cur != 0xffffffffu) buf[fphys(brev12(cur))] = c2(acc.x * alpha, acc.y * alpha);
            cur = n;
            acc = c2(v * wx, v * wy);
          } else {
            acc.x = fma(v, wx, acc.x);
            acc.y = fma(v, wy, acc.y);
          }
        }
      }
      if (cur != 0xffffffffu) buf[fphys(brev12(cur))] = c2(acc.x * alpha, acc.y * alpha);
    }
    __syncthreads();
    // ---- B side: imaginary part (i * w * v)
    {
      const double* row = a.matB + ((size_t)t * a.kc + kk) * a.SB;
      uint32_t cur = 0xffffffffu;
      double2 acc = c2(0.0, 0.0);
      for (int s0 = 0; s0 < cntB; s0 += kBatch) {
        double vv[kBatch];
        uint32_t hh[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          const bool ok = s0 + u < cntB;
          const int64_t e = (int64_t)(s0 + u) * kT + tid;
          vv[u] = ok ? __ldg(row + e) : 0.0;
          hh[u] = ok ? (uint32_t)codesB[e] : 0xffffffffu;
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          if (hh[u] == 0xffffffffu) break;
          const double v = vv[u];
          const uint32_t h = hh[u];
          const uint32_t n = h & (kFL - 1);
          double wx = 1.0, wy = 0.0;
          if (R > 1) {
            const uint32_t j = premixed ? (h >> kFLog) : (((h >> kFLog) * (uint32_t)r) & (uint32_t)(R - 1));
            if (j < 256) { wx = wRx[j]; wy = wRy[j]; }
            else { const double2 w = __ldg(tw + (j << kFLog)); wx = w.x; wy = w.y; }
          }
          // contribution i * w * v
          if (n != cur) {
            if (cur != 0xffffffffu) {
              double2& dst = buf[fphys(brev12(cur))];
              dst = c2(fma(acc.x, beta, dst.x), fma(acc.y, beta, dst.y));
            }
            cur = n;
            acc = c2(-v * wy, v * wx);
          } else {
            acc.x = fma(-v, wy, acc.x);
            acc.y = fma(v, wx, acc.y);
          }
        }
      }
      if (cur != 0xffffffffu) {
        double2& dst = buf[fphys(brev12(cur))];
        dst = c2(fma(acc.x, beta, dst.x), fma(acc.y, beta, dst.y));
      }
    }
    __syncthreads();
    // ---- pass 0 (stages 0-2) with the slab twiddle w_b^{n r}
    {
      const int base = tid * 8;
      double2 x[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) x[e] = buf[fphys(base + e)];
      if (R > 1) {
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const uint32_t n = brev12((uint32_t)(base + e));
          x[e] = cm(x[e], cm(ptHi[n >> 6], ptLo[n & 63]));
        }
      }
      r8_dit(x, c2(1.0, 0.0));
#pragma unroll
      for (int e = 0; e < 8; ++e) buf[fphys(base + e)] = x[e];
    }
    __syncthreads();
    // ---- passes 1, 2 (stages 3-5, 6-8)
#pragma unroll
    for (int p = 1; p <= 2; ++p) {
      const int s0 = 3 * p, half = 1 << s0;
      const int kk2 = tid & (half - 1);
      const int base = ((tid >> s0) << (s0 + 3)) | kk2;
      double2 x[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) x[e] = buf[fphys(base + e * half)];
      r8_dit(x, p == 1 ? tw1[kk2] : tw2[kk2]);
#pragma unroll
      for (int e = 0; e < 8; ++e) buf[fphys(base + e * half)] = x[e];
      __syncthreads();
    }
    // ---- pass 3 (stages 9-11): outputs m = tid + 512 e; Q += Z^2
    {
      double2 x[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) x[e] = buf[fphys(tid + 512 * e)];
      r8_dit(x, tw3[tid]);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        q[e].x = fma(x[e].x, x[e].x, fma(-x[e].y, x[e].y, q[e].x));
        q[e].y = fma(2.0 * x[e].x, x[e].y, q[e].y);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int e = 0; e < 8; ++e) part[tid + 512 * e] = q[e];
}

// ------------------------------------------------------------ WHT kernel
__device__ __forceinline__ void hbf(double& a, double& b) {
  const double u = a, v = b;
  a = u + v;
  b = u - v;
}

template <int M>
__device__ __forceinline__ void wht_reg(double (&x)[M]) {
#pragma unroll
  for (int h = 1; h < M; h <<= 1)
#pragma unroll
    for (int e = 0; e < M; ++e)
      if (!(e & h)) hbf(x[e], x[e + h]);
}

template <typename CodeT>
__global__ void __launch_bounds__(kT, 1) k_sketch_fwht_v1(V1Args a) {
  extern __shared__ __align__(16) unsigned char sm[];
  double* xs = reinterpret_cast<double*>(sm);
  double* ys = xs + kWPhys;
  CodeT* cA = reinterpret_cast<CodeT*>(ys + kWPhys);
  CodeT* cB = cA + (a.codes_in_smem ? a.SA : 0);
  const int tid = threadIdx.x;
  const int r = blockIdx.x, t = blockIdx.y, g = blockIdx.z;
  const int R = 1 << a.logR;
  const CodeT* gA = reinterpret_cast<const CodeT*>(a.codeA) + (size_t)t * a.SA;
  const CodeT* gB = reinterpret_cast<const CodeT*>(a.codeB) + (size_t)t * a.SB;
  // shared codes carry (n, parity of popc(q & r)) in bit kWLog
  if (a.codes_in_smem) {
    for (int64_t e = tid; e < a.SA; e += kT) {
      const uint32_t h = gA[e];
      cA[e] = (CodeT)((h & (kWL - 1)) | ((__popc((h >> kWLog) & (uint32_t)r) & 1u) << kWLog));
    }
    for (int64_t e = tid; e < a.SB; e += kT) {
      const uint32_t h = gB[e];
      cB[e] = (CodeT)((h & (kWL - 1)) | ((__popc((h >> kWLog) & (uint32_t)r) & 1u) << kWLog));
    }
  }
  const bool premixed = a.codes_in_smem != 0;
  const CodeT* codesA = a.codes_in_smem ? cA : gA;
  const CodeT* codesB = a.codes_in_smem ? cB : gB;
  const int cntA = (int)a.countA[(size_t)t * kT + tid];
  const int cntB = (int)a.countB[(size_t)t * kT + tid];
  double* part = reinterpret_cast<double*>(a.partial) + (((size_t)g * a.d + t) * (size_t)R + r) * kWL;
  double pacc[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int gi = tid + (e >> 3) * 512, ee = e & 7;  // output m = gi + 1024 ee
    pacc[e] = a.accumulate ? part[gi + 1024 * ee] : 0.0;
  }
  const int64_t per = (a.kc + a.G - 1) / a.G;
  const int64_t kb = (int64_t)g * per;
  const int64_t ke = kb + per < a.kc ? kb + per : a.kc;
  __syncthreads();
  for (int64_t kk = kb; kk < ke; ++kk) {
    for (int e = tid; e < kWPhys; e += kT) { xs[e] = 0.0; ys[e] = 0.0; }
    __syncthreads();
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const double* row = side == 0 ? a.matA + ((size_t)t * a.kc + kk) * a.SA
                                    : a.matB + ((size_t)t * a.kc + kk) * a.SB;
      const CodeT* codes = side == 0 ? codesA : codesB;
      double* dst = side == 0 ? xs : ys;
      const int cnt = side == 0 ? cntA : cntB;
      uint32_t cur = 0xffffffffu;
      double acc = 0.0;
      for (int s0 = 0; s0 < cnt; s0 += kBatch) {
        double vv[kBatch];
        uint32_t hh[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          const bool ok = s0 + u < cnt;
          const int64_t e = (int64_t)(s0 + u) * kT + tid;
          vv[u] = ok ? __ldg(row + e) : 0.0;
          hh[u] = ok ? (uint32_t)codes[e] : 0xffffffffu;
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          if (hh[u] == 0xffffffffu) break;
          const uint32_t h = hh[u];
          const uint32_t n = h & (kWL - 1);
          const uint32_t neg = premixed ? (h >> kWLog) : (__popc((h >> kWLog) & (uint32_t)r) & 1u);
          const double v = neg ? -vv[u] : vv[u];
          if (n != cur) {
            if (cur != 0xffffffffu) dst[wphys(cur)] = acc;
            cur = n;
            acc = v;
          } else {
            acc += v;
          }
        }
      }
      if (cur != 0xffffffffu) dst[wphys(cur)] = acc;
    }
    __syncthreads();
    // pass 0: radix-16 on points tid*16 + e (stages 0-3)
    {
      const int base = tid * 16;
      double x[16], y[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) { x[e] = xs[wphys(base + e)]; y[e] = ys[wphys(base + e)]; }
      wht_reg<16>(x);
      wht_reg<16>(y);
#pragma unroll
      for (int e = 0; e < 16; ++e) { xs[wphys(base + e)] = x[e]; ys[wphys(base + e)] = y[e]; }
    }
    __syncthreads();
    // passes 1, 2: radix-8 at s0 = 4, 7 (two groups per thread)
#pragma unroll
    for (int p = 1; p <= 2; ++p) {
      const int s0 = p == 1 ? 4 : 7, half = 1 << s0;
#pragma unroll
      for (int gg = 0; gg < 2; ++gg) {
        const int gi = tid + gg * 512;
        const int base = ((gi >> s0) << (s0 + 3)) | (gi & (half - 1));
        double x[8], y[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) { x[e] = xs[wphys(base + e * half)]; y[e] = ys[wphys(base + e * half)]; }
        wht_reg<8>(x);
        wht_reg<8>(y);
#pragma unroll
        for (int e = 0; e < 8; ++e) { xs[wphys(base + e * half)] = x[e]; ys[wphys(base + e * half)] = y[e]; }
      }
      __syncthreads();
    }
    // pass 3: radix-8 at s0 = 10; outputs m = gi + 1024 e; P += X * Y
#pragma unroll
    for (int gg = 0; gg < 2; ++gg) {
      const int gi = tid + gg * 512;
      double x[8], y[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) { x[e] = xs[wphys(gi + 1024 * e)]; y[e] = ys[wphys(gi + 1024 * e)]; }
      wht_reg<8>(x);
      wht_reg<8>(y);
#pragma unroll
      for (int e = 0; e < 8; ++e) pacc[gg * 8 + e] = fma(x[e], y[e], pacc[gg * 8 + e]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int gi = tid + (e >> 3) * 512, ee = e & 7;
    part[gi + 1024 * ee] = pacc[e];
  }
}

// ------------------------------------------------------------------ launch
SketchPlan plan_sketch_v1(int variant, int64_t n_a, int64_t n_inner, int64_t n_b, int d, int b,
                          int sms) {
  SketchPlan P{};
  P.variant = variant;
  P.d = d;
  P.b = b;
  P.log2b = 0;
  while ((1 << P.log2b) < b) ++P.log2b;
  P.logL = variant == kVariantFFT ? kFLog : kWLog;
  P.L = 1 << P.logL;
  P.logR = P.log2b - P.logL;
  P.R = 1 << P.logR;
  P.KB = 1;
  P.n_a = n_a;
  P.n_inner = n_inner;
  P.n_b = n_b;
  int64_t G = sms / ((int64_t)P.R * d);
  if (G < 1) G = 1;
  if (G > n_inner && n_inner > 0) G = n_inner;
  if (G > 65535) G = 65535;
  P.G = (int)G;
  return P;
}

bool sketch_v1_applicable(int variant, int b, int64_t n_a, int64_t n_b) {
  (void)n_a; (void)n_b;
  if (variant == kVariantFFT) return b >= kFL && b <= (1 << 20);
  return b >= kWL && b <= (1 << 21);
}

static size_t v1_smem(int variant, bool codes_in_smem, bool u16, int64_t SA, int64_t SB) {
  const size_t cb = u16 ? 2 : 4;
  const size_t codes = codes_in_smem ? (size_t)(SA + SB) * cb : 0;
  if (variant == kVariantFFT) return (size_t)(kFPhys + 64 + 64 + 8 + 64 + 512 + 256) * 16 + codes;
  return (size_t)2 * kWPhys * 8 + codes;
}

void launch_sketch_v1(const SketchPlan& SP, const SlabPlan& P, const double* dMatA,
                      const double* dMatB, int64_t kc, const int* dScaleExp, int64_t k0,
                      const double2* dTw, void* dPartial, int accumulate, cudaStream_t s) {
  V1Args a;
  a.matA = dMatA;
  a.matB = dMatB;
  a.codeA = P.codeA.ptr;
  a.codeB = P.codeB.ptr;
  a.countA = P.countA.as<uint32_t>();
  a.countB = P.countB.as<uint32_t>();
  a.scale_exp = dScaleExp;
  a.tw = dTw;
  a.partial = dPartial;
  a.SA = (int64_t)P.EA * kT;
  a.SB = (int64_t)P.EB * kT;
  a.kc = kc;
  a.k0 = k0;
  a.d = SP.d;
  a.log2b = SP.log2b;
  a.logR = SP.logR;
  a.G = SP.G;
  a.accumulate = accumulate;
  const size_t limit = 227 * 1024;
  bool in_smem = v1_smem(SP.variant, true, P.u16, a.SA, a.SB) <= limit;
  a.codes_in_smem = in_smem ? 1 : 0;
  const size_t smem = v1_smem(SP.variant, in_smem, P.u16, a.SA, a.SB);
  dim3 grid((unsigned)SP.R, (unsigned)SP.d, (unsigned)SP.G);
  ProfScope prof("sketch", s);
  count_launch();
  if (SP.variant == kVariantFFT) {
    if (P.u16) {
      CMM_CUDA(cudaFuncSetAttribute(k_sketch_fft_v1<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_sketch_fft_v1<uint16_t><<<grid, kT, smem, s>>>(a);
    } else {
      CMM_CUDA(cudaFuncSetAttribute(k_sketch_fft_v1<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_sketch_fft_v1<uint32_t><<<grid, kT, smem, s>>>(a);
    }
  } else {
    if (P.u16) {
      CMM_CUDA(cudaFuncSetAttribute(k_sketch_fwht_v1<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_sketch_fwht_v1<uint16_t><<<grid, kT, smem, s>>>(a);
    } else {
      CMM_CUDA(cudaFuncSetAttribute(k_sketch_fwht_v1<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_sketch_fwht_v1<uint32_t><<<grid, kT, smem, s>>>(a);
    }
  }
  CMM_CUDA(cudaGetLastError());
}

}  // namespace cmm
