// Mixed-precision sketch kernels (FP32 inputs; no reference twin: the
// reference binding is FP64-only, compmatmul.cpp:22-30).
//
// Same plan / materialization / slab decomposition as the v1 FP64 kernels,
// with L = 8192 frequencies per CTA and:
//  * FFT: the slab sequence and its radix-16/8 passes in FP32 (complex
//    float, padded shared layout); Q[f] += Z[f]^2 accumulated across k with
//    two-sum compensation (hi + lo FP32 pairs, Knuth's TwoSum); the pair is
//    summed in FP64 when the partial is written, so the k-group reduction
//    and the inverse transform stay FP64.
//  * FWHT: the first three Hadamard factors (H16 (x) H16 (x) H16 of
//    WHT_8192 = H2 (x) H16 (x) H16 (x) H16) run on the tensor cores as
//    16x16 +-1 products (mma.sync m16n8k16 BF16 -> FP32): each FP32 operand
//    is split into hi = bf16(x) and lo = bf16(x - hi), and H.x = H.hi + H.lo
//    is accumulated in FP32 (the +-1 products are exact).  The last radix-2
//    factor and P += X * Y run on the CUDA cores, P compensated like Q.
#include <cuda_bf16.h>

#include "cmm_internal.h"

namespace cmm {

constexpr int kMT = kPlanThreads;  // 512
constexpr int kML = 8192, kMLog = 13;
constexpr int kMBatch = 8;
constexpr int kMSkip = -0x7fffffff;

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 fcm(float2 a, float2 b) {
  return f2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 fcsq(float2 a) { return f2(fmaf(a.x, a.x, -a.y * a.y), 2.f * a.x * a.y); }
__device__ __forceinline__ void fbfly(float2& a, float2& b, float2 w) {
  const float2 t = fcm(b, w);
  b = f2(a.x - t.x, a.y - t.y);
  a = f2(a.x + t.x, a.y + t.y);
}
// Knuth TwoSum: hi + lo += x
__device__ __forceinline__ void two_sum_acc(float& hi, float& lo, float x) {
  const float s = hi + x;
  const float bp = s - hi;
  const float err = (hi - (s - bp)) + (x - bp);
  hi = s;
  lo += err;
}

// complex float, padded: phys(p) = p + p / 16 (8-byte elements)
__device__ __forceinline__ int mphys(int p) { return p + (p >> 4); }
constexpr int kMPhys = kML + kML / 16;

__device__ __forceinline__ void r8_dit_f(float2 (&x)[8], float2 W) {
  const float h = 0.70710678118654752440f;
  const float2 W2 = fcsq(W), W4 = fcsq(W2);
  fbfly(x[0], x[1], W4); fbfly(x[2], x[3], W4); fbfly(x[4], x[5], W4); fbfly(x[6], x[7], W4);
  const float2 W2m = f2(W2.y, -W2.x);
  fbfly(x[0], x[2], W2); fbfly(x[4], x[6], W2); fbfly(x[1], x[3], W2m); fbfly(x[5], x[7], W2m);
  const float2 W1 = fcm(W, f2(h, -h));
  const float2 Wi = f2(W.y, -W.x);
  const float2 W3 = fcm(W, f2(-h, -h));
  fbfly(x[0], x[4], W); fbfly(x[1], x[5], W1); fbfly(x[2], x[6], Wi); fbfly(x[3], x[7], W3);
}

// four radix-2 DIT stages on 16 consecutive points (twiddles w_{2^{i+1}}^{e mod 2^i})
__device__ __forceinline__ void r16_dit_first(float2 (&x)[16], const float2* w16) {
#pragma unroll
  for (int st = 0; st < 4; ++st) {
    const int h = 1 << st;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      if (e & h) continue;
      // twiddle w_{2h}^{e mod h} = w_16^{(e mod h) * 8 / h}
      const int k = (e & (h - 1)) * (8 >> st);
      fbfly(x[e], x[e + h], w16[k]);
    }
  }
}

struct MixArgs {
  const float* matA;
  const float* matB;
  const void* codeA;
  const void* codeB;
  const uint32_t* countA;
  const uint32_t* countB;
  const int* scale_exp;
  const double2* tw;
  void* partial;  // double2 (FFT) / double (FWHT) [g][t][r][L]
  int64_t SA, SB, kc, k0;
  int d, log2b, logR, G, accumulate, codes_in_smem;
};

__device__ __forceinline__ uint32_t brev13(uint32_t n) { return __brev(n) >> 19; }

template <typename CodeT>
__global__ void __launch_bounds__(kMT, 1) k_sketch_fft_f32(MixArgs a) {
  extern __shared__ __align__(16) unsigned char sm[];
  float2* buf = reinterpret_cast<float2*>(sm);
  float2* ptHi = buf + kMPhys;   // w_b^{64 x r}, x < 128
  float2* ptLo = ptHi + 128;     // w_b^{y r}, y < 64
  float2* tw1 = ptLo + 64;       // w_128^kk,  kk < 16
  float2* tw2 = tw1 + 16;        // w_1024^kk, kk < 128
  float2* tw3 = tw2 + 128;       // w_8192^kk, kk < 1024
  float2* w16 = tw3 + 1024;      // w_16^k, k < 8
  float* wRx = reinterpret_cast<float*>(w16 + 8);  // w_R^j, j < min(R, 256)
  float* wRy = wRx + 256;
  CodeT* cA = reinterpret_cast<CodeT*>(wRy + 256);
  CodeT* cB = cA + (a.codes_in_smem ? a.SA : 0);

  const int tid = threadIdx.x;
  const int r = blockIdx.x, t = blockIdx.y, g = blockIdx.z;
  const int R = 1 << a.logR;
  const double2* tw = a.tw;
  auto tf = [&](uint32_t i) { const double2 v = tw[i]; return f2((float)v.x, (float)v.y); };
  for (int e = tid; e < 128; e += kMT) {
    ptHi[e] = tf((uint32_t)(64 * e) * (uint32_t)r);
    tw2[e] = tf((uint32_t)e << (a.log2b - 10));
  }
  for (int e = tid; e < 64; e += kMT) ptLo[e] = tf((uint32_t)e * (uint32_t)r);
  for (int e = tid; e < 16; e += kMT) tw1[e] = tf((uint32_t)e << (a.log2b - 7));
  for (int e = tid; e < 1024; e += kMT) tw3[e] = tf((uint32_t)e << (a.log2b - 13));
  for (int e = tid; e < 8; e += kMT) w16[e] = tf((uint32_t)e << (a.log2b - 4));
  for (int e = tid; e < (R < 256 ? R : 256); e += kMT) {
    const float2 w = tf((uint32_t)e << kMLog);
    wRx[e] = w.x;
    wRy[e] = w.y;
  }
  const CodeT* gA = reinterpret_cast<const CodeT*>(a.codeA) + (size_t)t * a.SA;
  const CodeT* gB = reinterpret_cast<const CodeT*>(a.codeB) + (size_t)t * a.SB;
  if (a.codes_in_smem) {
    for (int64_t e = tid; e < a.SA; e += kMT) {
      const uint32_t h = gA[e];
      cA[e] = (CodeT)((h & (kML - 1)) | ((((h >> kMLog) * (uint32_t)r) & (uint32_t)(R - 1)) << kMLog));
    }
    for (int64_t e = tid; e < a.SB; e += kMT) {
      const uint32_t h = gB[e];
      cB[e] = (CodeT)((h & (kML - 1)) | ((((h >> kMLog) * (uint32_t)r) & (uint32_t)(R - 1)) << kMLog));
    }
  }
  const bool premixed = a.codes_in_smem != 0;
  const CodeT* codesA = a.codes_in_smem ? cA : gA;
  const CodeT* codesB = a.codes_in_smem ? cB : gB;
  const int cntA = (int)a.countA[(size_t)t * kMT + tid];
  const int cntB = (int)a.countB[(size_t)t * kMT + tid];

  // outputs of this thread: m = gi + 1024 e, gi in {tid, tid + 512}, e < 8
  double2* part = reinterpret_cast<double2*>(a.partial) + (((size_t)g * a.d + t) * (size_t)R + r) * kML;
  float qh[16][2], ql[16][2];
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int m = tid + (e >> 3) * 512 + 1024 * (e & 7);
    double2 v = a.accumulate ? part[m] : make_double2(0.0, 0.0);
    qh[e][0] = (float)v.x;
    ql[e][0] = (float)(v.x - (double)qh[e][0]);
    qh[e][1] = (float)v.y;
    ql[e][1] = (float)(v.y - (double)qh[e][1]);
  }
  const int64_t per = (a.kc + a.G - 1) / a.G;
  const int64_t kb = (int64_t)g * per;
  const int64_t ke = kb + per < a.kc ? kb + per : a.kc;
  __syncthreads();

  for (int64_t kk = kb; kk < ke; ++kk) {
    const int se = __ldg(a.scale_exp + a.k0 + kk);
    if (se == kMSkip) continue;
    for (int e = tid; e < kMPhys; e += kMT) buf[e] = f2(0.f, 0.f);
    const float alpha = __int_as_float((127 - se) << 23);
    const float beta = __int_as_float((127 + se) << 23);
    __syncthreads();
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const float* row = side == 0 ? a.matA + ((size_t)t * a.kc + kk) * a.SA
                                   : a.matB + ((size_t)t * a.kc + kk) * a.SB;
      const CodeT* codes = side == 0 ? codesA : codesB;
      const int cnt = side == 0 ? cntA : cntB;
      const float sc = side == 0 ? alpha : beta;
      uint32_t cur = 0xffffffffu;
      float2 acc = f2(0.f, 0.f);
      for (int s0 = 0; s0 < cnt; s0 += kMBatch) {
        float vv[kMBatch];
        uint32_t hh[kMBatch];
#pragma unroll
        for (int u = 0; u < kMBatch; ++u) {
          const bool ok = s0 + u < cnt;
          const int64_t e = (int64_t)(s0 + u) * kMT + tid;
          vv[u] = ok ? __ldg(row + e) : 0.f;
          hh[u] = ok ? (uint32_t)codes[e] : 0xffffffffu;
        }
#pragma unroll
        for (int u = 0; u < kMBatch; ++u) {
          if (hh[u] == 0xffffffffu) break;
          const float v = vv[u];
          const uint32_t h = hh[u];
          const uint32_t n = h & (kML - 1);
          float wx = 1.f, wy = 0.f;
          if (R > 1) {
            const uint32_t j = premixed ? (h >> kMLog) : (((h >> kMLog) * (uint32_t)r) & (uint32_t)(R - 1));
            if (j < 256) { wx = wRx[j]; wy = wRy[j]; }
            else { const double2 w = __ldg(tw + (j << kMLog)); wx = (float)w.x; wy = (float)w.y; }
          }
          // A side contributes w v to the real part, B side i w v
          const float cx = side == 0 ? v * wx : -v * wy;
          const float cy = side == 0 ? v * wy : v * wx;
          if (n != cur) {
            if (cur != 0xffffffffu) {
              float2& dst = buf[mphys(brev13(cur))];
              dst = side == 0 ? f2(acc.x * sc, acc.y * sc) : f2(fmaf(acc.x, sc, dst.x), fmaf(acc.y, sc, dst.y));
            }
            cur = n;
            acc = f2(cx, cy);
          } else {
            acc.x += cx;
            acc.y += cy;
          }
        }
      }
      if (cur != 0xffffffffu) {
        float2& dst = buf[mphys(brev13(cur))];
        dst = side == 0 ? f2(acc.x * sc, acc.y * sc) : f2(fmaf(acc.x, sc, dst.x), fmaf(acc.y, sc, dst.y));
      }
      __syncthreads();
    }
    // pass 0: radix-16 on points tid*16 + e with the slab twiddle
    {
      const int base = tid * 16;
      float2 x[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) x[e] = buf[mphys(base + e)];
      if (R > 1) {
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const uint32_t n = brev13((uint32_t)(base + e));
          x[e] = fcm(x[e], fcm(ptHi[n >> 6], ptLo[n & 63]));
        }
      }
      r16_dit_first(x, w16);
#pragma unroll
      for (int e = 0; e < 16; ++e) buf[mphys(base + e)] = x[e];
    }
    __syncthreads();
    // passes 1, 2: radix-8 at s0 = 4, 7 (two groups per thread)
#pragma unroll
    for (int p = 1; p <= 2; ++p) {
      const int s0 = p == 1 ? 4 : 7, half = 1 << s0;
#pragma unroll
      for (int gg = 0; gg < 2; ++gg) {
        const int gi = tid + gg * 512;
        const int kk2 = gi & (half - 1);
        const int base = ((gi >> s0) << (s0 + 3)) | kk2;
        float2 x[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) x[e] = buf[mphys(base + e * half)];
        r8_dit_f(x, p == 1 ? tw1[kk2] : tw2[kk2]);
#pragma unroll
        for (int e = 0; e < 8; ++e) buf[mphys(base + e * half)] = x[e];
      }
      __syncthreads();
    }
    // pass 3: radix-8 at s0 = 10; outputs m = gi + 1024 e; Q += Z^2 (two-sum)
#pragma unroll
    for (int gg = 0; gg < 2; ++gg) {
      const int gi = tid + gg * 512;
      float2 x[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) x[e] = buf[mphys(gi + 1024 * e)];
      r8_dit_f(x, tw3[gi]);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const float zr = fmaf(x[e].x, x[e].x, -x[e].y * x[e].y);
        const float zi = 2.f * x[e].x * x[e].y;
        two_sum_acc(qh[gg * 8 + e][0], ql[gg * 8 + e][0], zr);
        two_sum_acc(qh[gg * 8 + e][1], ql[gg * 8 + e][1], zi);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int m = tid + (e >> 3) * 512 + 1024 * (e & 7);
    part[m] = make_double2((double)qh[e][0] + (double)ql[e][0], (double)qh[e][1] + (double)ql[e][1]);
  }
}

// ---------------------------------------------------------------- FWHT
// fp32 buffers of 8192 points, padded phys(p) = p + p / 32
constexpr int kWPad = kML + kML / 32;
__device__ __forceinline__ int wph(int p) { return p + (p >> 5); }

__device__ __forceinline__ uint32_t pack_bf16(float lo_elem, float hi_elem) {
  // element with the lower column index goes to the low half
  const __nv_bfloat16 a = __float2bfloat16_rn(lo_elem);
  const __nv_bfloat16 b = __float2bfloat16_rn(hi_elem);
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

__device__ __forceinline__ void split_pair(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
  hi = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
  lo = pack_bf16(x0 - __bfloat162float(h0), x1 - __bfloat162float(h1));
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// One Hadamard-16 factor over the whole buffer: 512 vectors of 16 points,
// vector V, element e at point addr(V, e).  Each warp handles tiles of 16
// vectors; Y = X H16 with X split hi/lo (2 MMAs per 8-column half).
template <int STAGE>
__device__ __forceinline__ int hpoint(int V, int e) {
  if (STAGE == 0) return V * 16 + e;                       // stride 1
  if (STAGE == 1) return (V >> 4) * 256 + e * 16 + (V & 15);  // stride 16
  return (V >> 8) * 4096 + e * 256 + (V & 255);            // stride 256
}

template <int STAGE>
__device__ __forceinline__ void h16_stage(float* buf, const uint32_t (&hb)[2][2], int warp, int lane) {
  const int gq = lane >> 2, tq = lane & 3;
  for (int tile = warp; tile < 32; tile += kMT / 32) {
    const int V0 = tile * 16;
    // A fragment rows gq, gq+8; cols 2tq, 2tq+1, 2tq+8, 2tq+9
    float x[8];
    x[0] = buf[wph(hpoint<STAGE>(V0 + gq, 2 * tq))];
    x[1] = buf[wph(hpoint<STAGE>(V0 + gq, 2 * tq + 1))];
    x[2] = buf[wph(hpoint<STAGE>(V0 + gq + 8, 2 * tq))];
    x[3] = buf[wph(hpoint<STAGE>(V0 + gq + 8, 2 * tq + 1))];
    x[4] = buf[wph(hpoint<STAGE>(V0 + gq, 2 * tq + 8))];
    x[5] = buf[wph(hpoint<STAGE>(V0 + gq, 2 * tq + 9))];
    x[6] = buf[wph(hpoint<STAGE>(V0 + gq + 8, 2 * tq + 8))];
    x[7] = buf[wph(hpoint<STAGE>(V0 + gq + 8, 2 * tq + 9))];
    uint32_t ahi[4], alo[4];
    split_pair(x[0], x[1], ahi[0], alo[0]);
    split_pair(x[2], x[3], ahi[1], alo[1]);
    split_pair(x[4], x[5], ahi[2], alo[2]);
    split_pair(x[6], x[7], ahi[3], alo[3]);
    float c0[4] = {0.f, 0.f, 0.f, 0.f}, c1[4] = {0.f, 0.f, 0.f, 0.f};
    mma_bf16(c0, ahi, hb[0][0], hb[0][1]);
    mma_bf16(c0, alo, hb[0][0], hb[0][1]);
    mma_bf16(c1, ahi, hb[1][0], hb[1][1]);
    mma_bf16(c1, alo, hb[1][0], hb[1][1]);
    __syncwarp();
    // C fragment: rows gq, gq+8; cols 2tq, 2tq+1 (+8 for the second half)
    buf[wph(hpoint<STAGE>(V0 + gq, 2 * tq))] = c0[0];
    buf[wph(hpoint<STAGE>(V0 + gq, 2 * tq + 1))] = c0[1];
    buf[wph(hpoint<STAGE>(V0 + gq + 8, 2 * tq))] = c0[2];
    buf[wph(hpoint<STAGE>(V0 + gq + 8, 2 * tq + 1))] = c0[3];
    buf[wph(hpoint<STAGE>(V0 + gq, 2 * tq + 8))] = c1[0];
    buf[wph(hpoint<STAGE>(V0 + gq, 2 * tq + 9))] = c1[1];
    buf[wph(hpoint<STAGE>(V0 + gq + 8, 2 * tq + 8))] = c1[2];
    buf[wph(hpoint<STAGE>(V0 + gq + 8, 2 * tq + 9))] = c1[3];
  }
}

template <typename CodeT>
__global__ void __launch_bounds__(kMT, 1) k_sketch_fwht_tc(MixArgs a) {
  extern __shared__ __align__(16) unsigned char sm[];
  float* xs = reinterpret_cast<float*>(sm);
  float* ys = xs + kWPad;
  CodeT* cA = reinterpret_cast<CodeT*>(ys + kWPad);
  CodeT* cB = cA + (a.codes_in_smem ? a.SA : 0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r = blockIdx.x, t = blockIdx.y, g = blockIdx.z;
  const int R = 1 << a.logR;
  // B fragments of H16 (col-major 16x8 halves): b0,b1 = rows 2tq, 2tq+1 of
  // column gq; b2,b3 = rows 2tq+8, 2tq+9.  H[e][c] = (-1)^popc(e & c).
  uint32_t hb[2][2];
  {
    const int gq = lane >> 2, tq = lane & 3;
    auto h = [](int e, int c) { return (__popc(e & c) & 1) ? -1.f : 1.f; };
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int c = gq + 8 * half;
      hb[half][0] = pack_bf16(h(2 * tq, c), h(2 * tq + 1, c));
      hb[half][1] = pack_bf16(h(2 * tq + 8, c), h(2 * tq + 9, c));
    }
  }
  const CodeT* gA = reinterpret_cast<const CodeT*>(a.codeA) + (size_t)t * a.SA;
  const CodeT* gB = reinterpret_cast<const CodeT*>(a.codeB) + (size_t)t * a.SB;
  if (a.codes_in_smem) {
    for (int64_t e = tid; e < a.SA; e += kMT) {
      const uint32_t h = gA[e];
      cA[e] = (CodeT)((h & (kML - 1)) | ((__popc((h >> kMLog) & (uint32_t)r) & 1u) << kMLog));
    }
    for (int64_t e = tid; e < a.SB; e += kMT) {
      const uint32_t h = gB[e];
      cB[e] = (CodeT)((h & (kML - 1)) | ((__popc((h >> kMLog) & (uint32_t)r) & 1u) << kMLog));
    }
  }
  const bool premixed = a.codes_in_smem != 0;
  const CodeT* codesA = a.codes_in_smem ? cA : gA;
  const CodeT* codesB = a.codes_in_smem ? cB : gB;
  const int cntA = (int)a.countA[(size_t)t * kMT + tid];
  const int cntB = (int)a.countB[(size_t)t * kMT + tid];
  // outputs of this thread: m = tid + 512 e (e < 8) and m + 4096
  double* part = reinterpret_cast<double*>(a.partial) + (((size_t)g * a.d + t) * (size_t)R + r) * kML;
  float ph[16], pl[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int m = tid + 512 * (e & 7) + 4096 * (e >> 3);
    const double v = a.accumulate ? part[m] : 0.0;
    ph[e] = (float)v;
    pl[e] = (float)(v - (double)ph[e]);
  }
  const int64_t per = (a.kc + a.G - 1) / a.G;
  const int64_t kb = (int64_t)g * per;
  const int64_t ke = kb + per < a.kc ? kb + per : a.kc;
  __syncthreads();
  for (int64_t kk = kb; kk < ke; ++kk) {
    for (int e = tid; e < kWPad; e += kMT) { xs[e] = 0.f; ys[e] = 0.f; }
    __syncthreads();
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const float* row = side == 0 ? a.matA + ((size_t)t * a.kc + kk) * a.SA
                                   : a.matB + ((size_t)t * a.kc + kk) * a.SB;
      const CodeT* codes = side == 0 ? codesA : codesB;
      float* dst = side == 0 ? xs : ys;
      const int cnt = side == 0 ? cntA : cntB;
      uint32_t cur = 0xffffffffu;
      float acc = 0.f;
      for (int s0 = 0; s0 < cnt; s0 += kMBatch) {
        float vv[kMBatch];
        uint32_t hh[kMBatch];
#pragma unroll
        for (int u = 0; u < kMBatch; ++u) {
          const bool ok = s0 + u < cnt;
          const int64_t e = (int64_t)(s0 + u) * kMT + tid;
          vv[u] = ok ? __ldg(row + e) : 0.f;
          hh[u] = ok ? (uint32_t)codes[e] : 0xffffffffu;
        }
#pragma unroll
        for (int u = 0; u < kMBatch; ++u) {
          if (hh[u] == 0xffffffffu) break;
          const uint32_t h = hh[u];
          const uint32_t n = h & (kML - 1);
          const uint32_t neg = premixed ? (h >> kMLog) : (__popc((h >> kMLog) & (uint32_t)r) & 1u);
          const float v = neg ? -vv[u] : vv[u];
          if (n != cur) {
            if (cur != 0xffffffffu) dst[wph(cur)] = acc;
            cur = n;
            acc = v;
          } else {
            acc += v;
          }
        }
      }
      if (cur != 0xffffffffu) dst[wph(cur)] = acc;
    }
    __syncthreads();
    // three Hadamard-16 factors on the tensor cores, x and y
    h16_stage<0>(xs, hb, warp, lane);
    h16_stage<0>(ys, hb, warp, lane);
    __syncthreads();
    h16_stage<1>(xs, hb, warp, lane);
    h16_stage<1>(ys, hb, warp, lane);
    __syncthreads();
    h16_stage<2>(xs, hb, warp, lane);
    h16_stage<2>(ys, hb, warp, lane);
    __syncthreads();
    // last factor H2 (stride 4096) and P += X * Y (two-sum)
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int m = tid + 512 * e;
      const float x0 = xs[wph(m)], x1 = xs[wph(m + 4096)];
      const float y0 = ys[wph(m)], y1 = ys[wph(m + 4096)];
      two_sum_acc(ph[e], pl[e], (x0 + x1) * (y0 + y1));
      two_sum_acc(ph[e + 8], pl[e + 8], (x0 - x1) * (y0 - y1));
    }
    __syncthreads();
  }
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int m = tid + 512 * (e & 7) + 4096 * (e >> 3);
    part[m] = (double)ph[e] + (double)pl[e];
  }
}

// ------------------------------------------------------------------ launch
SketchPlan plan_sketch_mixed(int variant, int64_t n_a, int64_t n_inner, int64_t n_b, int d, int b,
                             int sms) {
  SketchPlan P{};
  P.variant = variant;
  P.d = d;
  P.b = b;
  P.log2b = 0;
  while ((1 << P.log2b) < b) ++P.log2b;
  P.logL = kMLog;
  P.L = kML;
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

bool sketch_mixed_applicable(int variant, int b) {
  (void)variant;
  return b >= kML && b <= (1 << 21);
}

static size_t mixed_smem(int variant, bool codes_in_smem, bool u16, int64_t SA, int64_t SB) {
  const size_t cb = u16 ? 2 : 4;
  const size_t codes = codes_in_smem ? (size_t)(SA + SB) * cb : 0;
  if (variant == kVariantFFT)
    return (size_t)(kMPhys + 128 + 64 + 16 + 128 + 1024 + 8) * 8 + 512 * 4 + codes;
  return (size_t)2 * kWPad * 4 + codes;
}

void launch_sketch_mixed(const SketchPlan& SP, const SlabPlan& P, const float* dMatA,
                         const float* dMatB, int64_t kc, const int* dScaleExp, int64_t k0,
                         const double2* dTw, void* dPartial, int accumulate, cudaStream_t s) {
  MixArgs a;
  a.matA = dMatA;
  a.matB = dMatB;
  a.codeA = P.codeA.ptr;
  a.codeB = P.codeB.ptr;
  a.countA = P.countA.as<uint32_t>();
  a.countB = P.countB.as<uint32_t>();
  a.scale_exp = dScaleExp;
  a.tw = dTw;
  a.partial = dPartial;
  a.SA = (int64_t)P.EA * kMT;
  a.SB = (int64_t)P.EB * kMT;
  a.kc = kc;
  a.k0 = k0;
  a.d = SP.d;
  a.log2b = SP.log2b;
  a.logR = SP.logR;
  a.G = SP.G;
  a.accumulate = accumulate;
  const size_t limit = 227 * 1024;
  const bool in_smem = mixed_smem(SP.variant, true, P.u16, a.SA, a.SB) <= limit;
  a.codes_in_smem = in_smem ? 1 : 0;
  const size_t smem = mixed_smem(SP.variant, in_smem, P.u16, a.SA, a.SB);
  dim3 grid((unsigned)SP.R, (unsigned)SP.d, (unsigned)SP.G);
  ProfScope prof("sketch", s);
  count_launch();
#define CMM_MIX_LAUNCH(K, T)                                                                    \
  do {                                                                                          \
    CMM_CUDA(cudaFuncSetAttribute(K<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    K<T><<<grid, kMT, smem, s>>>(a);                                                            \
  } while (0)
  if (SP.variant == kVariantFFT) {
    if (P.u16) CMM_MIX_LAUNCH(k_sketch_fft_f32, uint16_t);
    else CMM_MIX_LAUNCH(k_sketch_fft_f32, uint32_t);
  } else {
    if (P.u16) CMM_MIX_LAUNCH(k_sketch_fwht_tc, uint16_t);
    else CMM_MIX_LAUNCH(k_sketch_fwht_tc, uint32_t);
  }
#undef CMM_MIX_LAUNCH
  CMM_CUDA(cudaGetLastError());
}

// ------------------------------------------------- fp32 row scale / rows
__device__ __forceinline__ int expo_of_f(float m) { return (int)((__float_as_int(m) >> 23) & 0xff) - 127; }

__global__ void k_row_scale_f32(const float* AT, const float* B, int64_t n_a, int64_t n_b, int* out) {
  const int64_t k = blockIdx.x;
  const float* ra = AT + k * n_a;
  const float* rb = B + k * n_b;
  float ma = 0.f, mb = 0.f;
  for (int64_t i = threadIdx.x; i < n_a; i += blockDim.x) ma = fmaxf(ma, fabsf(__ldg(ra + i)));
  for (int64_t j = threadIdx.x; j < n_b; j += blockDim.x) mb = fmaxf(mb, fabsf(__ldg(rb + j)));
  for (int o = 16; o > 0; o >>= 1) {
    ma = fmaxf(ma, __shfl_xor_sync(0xffffffffu, ma, o));
    mb = fmaxf(mb, __shfl_xor_sync(0xffffffffu, mb, o));
  }
  __shared__ float sa[32], sb[32];
  if ((threadIdx.x & 31) == 0) { sa[threadIdx.x >> 5] = ma; sb[threadIdx.x >> 5] = mb; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) { ma = fmaxf(ma, sa[i]); mb = fmaxf(mb, sb[i]); }
    int e;
    if (!(ma > 0.f) || !(mb > 0.f)) e = (ma == 0.f || mb == 0.f) ? kMSkip : 0;
    else {
      e = (expo_of_f(ma) - expo_of_f(mb)) / 2;
      e = e > 60 ? 60 : (e < -60 ? -60 : e);
    }
    out[k] = e;
  }
}

void launch_row_scale_f32(const float* dAT, const float* dB, int64_t n_a, int64_t n_inner,
                          int64_t n_b, int* dScaleExp, cudaStream_t s) {
  if (n_inner <= 0) return;
  ProfScope prof("scale", s);
  count_launch();
  k_row_scale_f32<<<(unsigned)n_inner, 256, 0, s>>>(dAT, dB, n_a, n_b, dScaleExp);
  CMM_CUDA(cudaGetLastError());
}

// materialize fp32 rows (same slot layout as the FP64 path)
// FP32 copies of the rows in slot order, as k_materialize: 1024 threads
// per inner index, four consecutive slots per thread (one 16-byte index
// load, one 16-byte streaming store)
__global__ void __launch_bounds__(1024) k_materialize_f32(const float* __restrict__ AT,
                                                         const float* __restrict__ B, int64_t n_a,
                                                         int64_t n_b, int64_t k0, int d,
                                                         const uint32_t* __restrict__ srcA,
                                                         const uint32_t* __restrict__ srcB, int64_t SA,
                                                         int64_t SB, int64_t kc, float* __restrict__ outA,
                                                         float* __restrict__ outB, int stage) {
  extern __shared__ float srowf[];
  const int64_t kk = blockIdx.x;
  for (int side = 0; side < 2; ++side) {
    const int64_t N = side == 0 ? n_a : n_b;
    const int64_t S = side == 0 ? SA : SB;
    const float* row = (side == 0 ? AT : B) + (size_t)(k0 + kk) * N;
    const uint32_t* src = side == 0 ? srcA : srcB;
    float* out = side == 0 ? outA : outB;
    if (stage) {
      for (int64_t i = threadIdx.x; i < N; i += blockDim.x) srowf[i] = __ldg(row + i);
      __syncthreads();
    }
    for (int t = 0; t < d; ++t) {
      const uint4* st = reinterpret_cast<const uint4*>(src + (size_t)t * S);
      float4* ot = reinterpret_cast<float4*>(out + ((size_t)t * kc + kk) * S);
      for (int64_t q = threadIdx.x; q < S / 4; q += blockDim.x) {
        const uint4 sv = __ldg(st + q);
        const uint32_t svs[4] = {sv.x, sv.y, sv.z, sv.w};
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          v[u] = 0.f;
          if (svs[u] != kPadSlot) {
            v[u] = stage ? srowf[svs[u] & 0x7fffffffu] : __ldg(row + (svs[u] & 0x7fffffffu));
            if (!(svs[u] >> 31)) v[u] = -v[u];
          }
        }
        __stcs(ot + q, make_float4(v[0], v[1], v[2], v[3]));
      }
    }
    __syncthreads();
  }
}

void launch_materialize_f32(const SlabPlan& P, const float* dAT, const float* dB, int64_t k0,
                            int64_t kc, float* dOutA, float* dOutB, cudaStream_t s) {
  if (kc <= 0) return;
  const int64_t nmax = P.n_a > P.n_b ? P.n_a : P.n_b;
  const size_t smem = (size_t)nmax * 4;
  const int stage = smem <= 200 * 1024 ? 1 : 0;
  const int64_t SA = P.slots_a(), SB = P.slots_b();
  if (SA % 4 || SB % 4) throw runtime_error("materialize: segment slots must be a multiple of 4");
  ProfScope prof("materialize", s);
  count_launch();
  if (stage)
    CMM_CUDA(cudaFuncSetAttribute(k_materialize_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_materialize_f32<<<(unsigned)kc, 1024, stage ? smem : 0, s>>>(dAT, dB, P.n_a, P.n_b, k0, P.d,
                                                                P.srcA.as<uint32_t>(), P.srcB.as<uint32_t>(),
                                                                SA, SB, kc, dOutA, dOutB, stage);
  CMM_CUDA(cudaGetLastError());
}

}  // namespace cmm
