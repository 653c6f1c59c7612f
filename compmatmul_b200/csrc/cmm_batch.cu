// Batched products: many independent compressed products of uneven shape in
// ONE persistent sketch launch (work queue), the whole per-batch sequence
// captured in a CUDA graph, and an autotuner for the per-product slab length
// and transform radix.
//
// Work item = (product, repetition t, frequency slab r, k-group g).  One CTA
// of kBT threads takes an item from a device counter and, for every inner
// index k of its group, count-sketches row k of AT and of B into its slab
// (decimation in frequency as in the slab kernels: bucket h goes to
// position h mod L with weight w_b^{h r} for the FFT, (-1)^{popc((h div L)
// & r)} for the FWHT), transforms the slab in shared memory and accumulates
// Z^2 (FFT, packed z = alpha x + i beta y) or X Y (FWHT) for its L
// frequencies in registers.  The partials land in the slab layout
// [g][t][r][m] that the existing k-group reduction + inverse (launch_finalize)
// reads, so each product then finishes exactly like a single product.
//
// Precision: Real = double (plain FP64) or float (mixed: FP32 data and
// transforms, two-sum compensated accumulation across k, FWHT Hadamard-16
// stages on the tensor cores as BF16 hi/mid/lo products, FP64 partials,
// reduction and inverse).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/compmatmul_b200.h"
#include "cmm_batch.h"
#include "cmm_fft_device.cuh"

namespace cmm {
namespace {

constexpr int kBT = 1024;        // threads per CTA
constexpr int kBFftLog = kBatchFftLog;
constexpr int kBWhtLog = kBatchWhtLog;
constexpr int kBSkip = -0x7fffffff;

using namespace dev;

__device__ __forceinline__ uint32_t brev_bits(uint32_t x, int lg) { return lg ? __brev(x) >> (32 - lg) : 0u; }

// padded shared layouts (one spare slot per 128 bytes): strided passes and
// consecutive sweeps touch distinct banks
template <int ES>
__device__ __forceinline__ int ph(int x) {
  return ES == 16 ? x + (x >> 3) : (ES == 8 ? x + (x >> 4) : x + (x >> 5));
}
template <int ES>
__host__ __device__ constexpr int ph_len(int L) {
  return ES == 16 ? L + L / 8 : (ES == 8 ? L + L / 16 : L + L / 32);
}

// one DIT pass of radix K over L points (bit-reversed in); wt[j] = w_4096^j.
// The first pass (s = 0, all twiddles trivial) adds side B's sub-sequence on
// load and clears it for the next row.
template <int K, bool FIRST, typename C>
__device__ __forceinline__ void fft_pass(C* buf, C* add, int L, int s, const C* wt, int ti, int nt) {
  constexpr int ES = (int)sizeof(C);
  constexpr int LK = K == 8 ? 3 : (K == 4 ? 2 : 1);
  const int half = 1 << s;
  for (int p = ti; p < (L >> LK); p += nt) {
    const int kk = p & (half - 1);
    const int base = ((p >> s) << (s + LK)) | kk;
    C x[K];
#pragma unroll
    for (int e = 0; e < K; ++e) x[e] = buf[ph<ES>(base + e * half)];
    if constexpr (FIRST) {
#pragma unroll
      for (int e = 0; e < K; ++e) {
        C* q = add + ph<ES>(base + e * half);
        const C y = *q;
        *q = mk(decltype(y.x)(0), decltype(y.x)(0));
        x[e] = mk(x[e].x + y.x, x[e].y + y.y);
      }
      if constexpr (K == 8) r8_first(x);
      else if constexpr (K == 4) r4_first(x);
      else add_sub(x[0], x[1]);
    } else {
      const C W = wt[kk << (kBFftLog - s - LK)];  // w_{K half}^kk
      if constexpr (K == 8) r8(x, W);
      else if constexpr (K == 4) r4(x, W);
      else bf(x[0], x[1], W);
    }
#pragma unroll
    for (int e = 0; e < K; ++e) buf[ph<ES>(base + e * half)] = x[e];
  }
}
// padded address of x + e * half for the compile-time stride HALF: linear
// in e once HALF is a multiple of the padding period
template <int ES, int HALF>
__device__ __forceinline__ int ph_step(int base, int e) {
  constexpr int P = ES == 16 ? 8 : (ES == 8 ? 16 : 32);  // elements per padding slot
  if constexpr (HALF % P == 0) return ph<ES>(base) + e * (HALF + HALF / P);
  else return ph<ES>(base + e * HALF);
}

// fft_pass with the slab length, stage and thread count fixed at compile
// time (the common slabs): every index is a constant offset from one base
template <int K, bool FIRST, int LOGL, int S, int NT, typename C>
__device__ __forceinline__ void fft_pass_fixed(C* buf, C* add, const C* wt, int ti) {
  constexpr int ES = (int)sizeof(C);
  constexpr int LK = K == 8 ? 3 : (K == 4 ? 2 : 1);
  constexpr int HALF = 1 << S;
  constexpr int GROUPS = (1 << LOGL) >> LK;
#pragma unroll
  for (int p0 = 0; p0 < GROUPS; p0 += NT) {
    const int p = p0 + ti;
    if (GROUPS % NT != 0 && p >= GROUPS) break;
    const int kk = p & (HALF - 1);
    const int base = ((p >> S) << (S + LK)) | kk;
    C x[K];
#pragma unroll
    for (int e = 0; e < K; ++e) x[e] = buf[ph_step<ES, HALF>(base, e)];
    if constexpr (FIRST) {
#pragma unroll
      for (int e = 0; e < K; ++e) {
        C* q = add + ph_step<ES, HALF>(base, e);
        const C y = *q;
        *q = mk(decltype(y.x)(0), decltype(y.x)(0));
        x[e] = mk(x[e].x + y.x, x[e].y + y.y);
      }
      if constexpr (K == 8) r8_first(x);
      else if constexpr (K == 4) r4_first(x);
      else add_sub(x[0], x[1]);
    } else {
      const C W = wt[kk << (kBFftLog - S - LK)];
      if constexpr (K == 8) r8(x, W);
      else if constexpr (K == 4) r4(x, W);
      else bf(x[0], x[1], W);
    }
#pragma unroll
    for (int e = 0; e < K; ++e) buf[ph_step<ES, HALF>(base, e)] = x[e];
  }
}

template <int K, int LOGL, int S, int NT, typename R>
__device__ __forceinline__ void wht_pass_fixed(R* arr, int ti) {
  constexpr int ES = (int)sizeof(R);
  constexpr int LK = K == 8 ? 3 : (K == 4 ? 2 : 1);
  constexpr int HALF = 1 << S;
  constexpr int GROUPS = (1 << LOGL) >> LK;
#pragma unroll
  for (int p0 = 0; p0 < GROUPS; p0 += NT) {
    const int p = p0 + ti;
    if (GROUPS % NT != 0 && p >= GROUPS) break;
    const int base = ((p >> S) << (S + LK)) | (p & (HALF - 1));
    R x[K];
#pragma unroll
    for (int e = 0; e < K; ++e) x[e] = arr[ph_step<ES, HALF>(base, e)];
    whtr<R, K>(x);
#pragma unroll
    for (int e = 0; e < K; ++e) arr[ph_step<ES, HALF>(base, e)] = x[e];
  }
}

// one natural-order WHT pass of radix K over L points
template <int K, typename R>
__device__ __forceinline__ void wht_pass(R* arr, int L, int s, int ti, int nt) {
  constexpr int ES = (int)sizeof(R);
  constexpr int LK = K == 8 ? 3 : (K == 4 ? 2 : 1);
  const int half = 1 << s;
  for (int p = ti; p < (L >> LK); p += nt) {
    const int base = ((p >> s) << (s + LK)) | (p & (half - 1));
    R x[K];
#pragma unroll
    for (int e = 0; e < K; ++e) x[e] = arr[ph<ES>(base + e * half)];
    whtr<R, K>(x);
#pragma unroll
    for (int e = 0; e < K; ++e) arr[ph<ES>(base + e * half)] = x[e];
  }
}

// ---------------------------------------------- tensor-core Hadamard-16
__device__ __forceinline__ uint32_t bf16x2(float lo_e, float hi_e) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo_e)) |
         ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi_e)) << 16);
}
// x = hi + mid + lo in BF16 (8 + 8 + 8 significant bits cover FP32's 24),
// so the +-1 products on the tensor cores lose nothing before the FP32
// accumulation
__device__ __forceinline__ void split3(float x0, float x1, uint32_t& hi, uint32_t& mid, uint32_t& lo) {
  const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
  const float r0 = x0 - __bfloat162float(h0), r1 = x1 - __bfloat162float(h1);
  const __nv_bfloat16 m0 = __float2bfloat16_rn(r0), m1 = __float2bfloat16_rn(r1);
  hi = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
  mid = (uint32_t)__bfloat16_as_ushort(m0) | ((uint32_t)__bfloat16_as_ushort(m1) << 16);
  lo = bf16x2(r0 - __bfloat162float(m0), r1 - __bfloat162float(m1));
}
__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// Hadamard-16 over bits [sh, sh + 4) of the index, L / 16 vectors in
// tiles of 16 (three m16n8k16 products per output half: hi, mid, lo);
// needs L >= 256
__device__ __forceinline__ void h16_stage(float* buf, int L, int sh, const uint32_t (&hb)[2][2],
                                          int warp, int lane, int nwarps) {
  const int gq = lane >> 2, tq = lane & 3;
  const int low = (1 << sh) - 1;
  auto hp = [&](int V, int e) { return ((V >> sh) << (sh + 4)) | (e << sh) | (V & low); };
  for (int tile = warp; tile < (L >> 8); tile += nwarps) {
    const int V0 = tile * 16;
    const int p[8] = {hp(V0 + gq, 2 * tq),     hp(V0 + gq, 2 * tq + 1),
                      hp(V0 + gq + 8, 2 * tq), hp(V0 + gq + 8, 2 * tq + 1),
                      hp(V0 + gq, 2 * tq + 8), hp(V0 + gq, 2 * tq + 9),
                      hp(V0 + gq + 8, 2 * tq + 8), hp(V0 + gq + 8, 2 * tq + 9)};
    float x[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) x[e] = buf[ph<4>(p[e])];
    uint32_t ahi[4], amid[4], alo[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) split3(x[2 * e], x[2 * e + 1], ahi[e], amid[e], alo[e]);
    float c0[4] = {0.f, 0.f, 0.f, 0.f}, c1[4] = {0.f, 0.f, 0.f, 0.f};
    mma16816(c0, alo, hb[0][0], hb[0][1]);  // smallest parts first
    mma16816(c0, amid, hb[0][0], hb[0][1]);
    mma16816(c0, ahi, hb[0][0], hb[0][1]);
    mma16816(c1, alo, hb[1][0], hb[1][1]);
    mma16816(c1, amid, hb[1][0], hb[1][1]);
    mma16816(c1, ahi, hb[1][0], hb[1][1]);
    const float y[8] = {c0[0], c0[1], c0[2], c0[3], c1[0], c1[1], c1[2], c1[3]};
#pragma unroll
    for (int e = 0; e < 8; ++e) buf[ph<4>(p[e])] = y[e];
  }
}

}  // namespace

template <typename Real>
__global__ void __launch_bounds__(kBT, 1)
    k_batch_sketch(const BProd* __restrict__ prods, const BItem* __restrict__ items, int n_items,
                   int* __restrict__ counter, const double2* __restrict__ tw4096) {
  using C = typename std::conditional<sizeof(Real) == 4, float2, double2>::type;
  constexpr bool kF32 = sizeof(Real) == 4;
  // rows per iteration: FP32 transforms two rows side by side (one half of
  // the CTA each), which fills every thread in the passes and halves the
  // barriers per row; FP64 slabs leave room for one row only
  constexpr int KB = kF32 ? 2 : 1;
  constexpr int NT = kBT / KB;  // threads per row
  constexpr int EC = (int)sizeof(C), ER = (int)sizeof(Real);
  constexpr int PLF = ph_len<EC>(1 << kBFftLog), PLW = ph_len<ER>(1 << kBWhtLog);
  constexpr size_t kSeq = 2 * PLF * sizeof(C) > 2 * PLW * sizeof(Real) ? 2 * PLF * sizeof(C) : 2 * PLW * sizeof(Real);
  extern __shared__ __align__(16) unsigned char sm[];
  const int tid = threadIdx.x, lane = tid & 31;
  const int q = tid / NT, ti = tid % NT;  // this thread's row slot and its index within it
  C* wt = reinterpret_cast<C*>(sm + KB * kSeq);  // pass twiddles w_4096^j, j < 4096
  C* dh = wt + (1 << kBFftLog);                  // DIF weights w_b^x = dh[x >> sd] * dl[x & (2^sd - 1)]
  C* dl = dh + 256;                              //   (b <= 2^16; larger b reads the global table)
  // row slot qq: FFT sides A, B (A also holds the transform); FWHT x, y
  auto bufA = [&](int qq) { return reinterpret_cast<C*>(sm + qq * kSeq); };
  auto bufB = [&](int qq) { return reinterpret_cast<C*>(sm + qq * kSeq) + PLF; };
  auto xsq = [&](int qq) { return reinterpret_cast<Real*>(sm + qq * kSeq); };
  auto ysq = [&](int qq) { return reinterpret_cast<Real*>(sm + qq * kSeq) + PLW; };
  __shared__ int s_item, s_log2b;
  for (int j = tid; j < (1 << kBFftLog); j += kBT) wt[j] = mk((Real)tw4096[j].x, (Real)tw4096[j].y);
  // every row slot starts clear; the passes and the accumulation clear what
  // they consume, so the slots are clear again before each row's scatter
  for (size_t e = tid * 16; e < KB * kSeq; e += kBT * 16)
    *reinterpret_cast<uint4*>(sm + e) = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) s_log2b = -1;
  uint32_t hb[2][2] = {{0u, 0u}, {0u, 0u}};
  if (kF32) {
    const int gq = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int hf = 0; hf < 2; ++hf) {
      const int c = gq + 8 * hf;
      auto hv = [](int e, int cc) { return (__popc(e & cc) & 1) ? -1.f : 1.f; };
      hb[hf][0] = bf16x2(hv(2 * tq, c), hv(2 * tq + 1, c));
      hb[hf][1] = bf16x2(hv(2 * tq + 8, c), hv(2 * tq + 9, c));
    }
  }

  for (;;) {
    __syncthreads();  // the previous item is finished and s_item is free
    if (tid == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const BItem I = items[it];
    const BProd P = prods[I.prod];
    const int logL = P.logL, L = 1 << logL, R = 1 << P.logR;
    const int sd = (P.log2b + 1) >> 1;  // split of the DIF weight index
    const bool fft = P.variant == kVariantFFT;
    const bool dtab = fft && P.log2b <= 16;
    if (dtab && s_log2b != P.log2b) {  // uniform: every thread reads the same s_log2b
      __syncthreads();
      for (int j = tid; j < (1 << (P.log2b - sd)); j += kBT) dh[j] = mk((Real)P.tw[j << sd].x, (Real)P.tw[j << sd].y);
      for (int j = tid; j < (1 << sd); j += kBT) dl[j] = mk((Real)P.tw[j].x, (Real)P.tw[j].y);
      __syncthreads();
      if (tid == 0) s_log2b = P.log2b;
    }
    const int64_t per = (P.n_inner + P.G - 1) / P.G;
    const int64_t kb = (int64_t)I.g * per;
    const int64_t ke = kb + per < P.n_inner ? kb + per : P.n_inner;
    const uint32_t r = (uint32_t)I.r;
    const uint32_t bmask = (1u << P.log2b) - 1u;
    // this thread's runs of whole buckets: cut index lt; with two rows per
    // iteration each thread takes both sides of its row, with one row
    // threads [0, 512) take side A and [512, 1024) side B
    const int lt = (KB == 2 ? ti : tid) & (kPlanThreads - 1);
    const int side0 = KB == 2 ? 0 : (tid >= kPlanThreads ? 1 : 0);
    const int side1 = KB == 2 ? 1 : side0;
    Real acc[8], lo[8];  // FFT: Re/Im of 4 frequencies; FWHT: 8 frequencies
#pragma unroll
    for (int j = 0; j < 8; ++j) { acc[j] = (Real)0; lo[j] = (Real)0; }
    const bool tc = kF32 && !fft && logL >= 8 && P.tc;  // Hadamard-16 stages on the tensor cores

    for (int64_t k0 = kb; k0 < ke; k0 += KB) {
      const int64_t k = k0 + q;
      int se = 0;
      bool live = k < ke;
      if (fft && live) {
        se = __ldg(P.scale + k);
        live = se != kBSkip;  // a zero row: the slot stays zero and adds nothing
      }
      // ---- count sketch + DIF split: one store per bucket (no atomics)
      if (live) {
        for (int side = side0; side <= side1; ++side) {
          const uint32_t* cut = (side ? P.cutB : P.cutA) + (size_t)I.t * (kPlanThreads + 1);
          const int beg = (int)__ldg(cut + lt), end = (int)__ldg(cut + lt + 1);
          const size_t seg = (size_t)I.t * (size_t)(side ? P.SB : P.SA);
          const uint32_t* src = (side ? P.srcB : P.srcA) + seg;
          const uint16_t* c16 = reinterpret_cast<const uint16_t*>(side ? P.codeB : P.codeA) + seg;
          const uint32_t* c32 = reinterpret_cast<const uint32_t*>(side ? P.codeB : P.codeA) + seg;
          const Real* row = reinterpret_cast<const Real*>(side ? P.B : P.AT) + (size_t)k * (size_t)(side ? P.n_b : P.n_a);
          uint32_t cur = 0xffffffffu;
          if (fft) {
            // A: alpha x, B: i beta y (alpha beta = 1), summed in the first pass
            const int e2 = side ? se : -se;
            const Real sc = kF32 ? (Real)__int_as_float((127 + e2) << 23)
                                 : (Real)__longlong_as_double((long long)(1023 + e2) << 52);
            C* arr = side ? bufB(q) : bufA(q);
            C run = mk((Real)0, (Real)0);
            for (int sl = beg; sl < end; ++sl) {
              const uint32_t sv = __ldg(src + sl);
              const uint32_t h = P.code16 ? (uint32_t)__ldg(c16 + sl) : __ldg(c32 + sl);
              Real v = __ldg(row + (sv & 0x7fffffffu)) * sc;
              if (!(sv >> 31)) v = -v;
              C c;
              if (r == 0) {
                c = mk(v, (Real)0);
              } else {
                const uint32_t x = (h * r) & bmask;
                C w;
                if (dtab) w = cmul(dh[x >> sd], dl[x & ((1u << sd) - 1u)]);
                else { const double2 g = __ldg(P.tw + x); w = mk((Real)g.x, (Real)g.y); }
                c = mk(v * w.x, v * w.y);
              }
              if (side) c = mk(-c.y, c.x);  // times i
              const uint32_t m = h & (uint32_t)(L - 1);
              if (m != cur) {
                if (cur != 0xffffffffu) arr[ph<EC>(brev_bits(cur, logL))] = run;
                cur = m;
                run = c;
              } else {
                run = mk(run.x + c.x, run.y + c.y);
              }
            }
            if (cur != 0xffffffffu) arr[ph<EC>(brev_bits(cur, logL))] = run;
          } else {
            Real* arr = side ? ysq(q) : xsq(q);
            Real run = (Real)0;
            for (int sl = beg; sl < end; ++sl) {
              const uint32_t sv = __ldg(src + sl);
              const uint32_t h = P.code16 ? (uint32_t)__ldg(c16 + sl) : __ldg(c32 + sl);
              Real v = __ldg(row + (sv & 0x7fffffffu));
              // sign(+-1) * (-1)^{popc(q & r)}: negate when the parity bit differs
              if (((sv >> 31) ^ 1u) ^ (__popc((h >> logL) & r) & 1u)) v = -v;
              const uint32_t m = h & (uint32_t)(L - 1);
              if (m != cur) {
                if (cur != 0xffffffffu) arr[ph<ER>((int)cur)] = run;
                cur = m;
                run = v;
              } else {
                run += v;
              }
            }
            if (cur != 0xffffffffu) arr[ph<ER>((int)cur)] = run;
          }
        }
      }
      __syncthreads();
      // ---- transform of this thread's row slot
      if (fft) {
        C* A = bufA(q);
        C* Bq = bufB(q);
        int s = 0;
        if (logL == 12 && P.radix == 8) {  // the common slab: strides fixed at compile time
          fft_pass_fixed<8, true, 12, 0, NT>(A, Bq, wt, ti);
          __syncthreads();
          fft_pass_fixed<8, false, 12, 3, NT>(A, Bq, wt, ti);
          __syncthreads();
          fft_pass_fixed<8, false, 12, 6, NT>(A, Bq, wt, ti);
          __syncthreads();
          fft_pass_fixed<8, false, 12, 9, NT>(A, Bq, wt, ti);
          __syncthreads();
          s = logL;
        } else if (P.radix == 8 && logL >= 3) fft_pass<8, true>(A, Bq, L, 0, wt, ti, NT), s = 3;
        else if (logL >= 2) fft_pass<4, true>(A, Bq, L, 0, wt, ti, NT), s = 2;
        else fft_pass<2, true>(A, Bq, L, 0, wt, ti, NT), s = 1;
        if (s < logL || !(logL == 12 && P.radix == 8)) __syncthreads();
        if (P.radix == 8)
          for (; s + 3 <= logL; s += 3) { fft_pass<8, false>(A, Bq, L, s, wt, ti, NT); __syncthreads(); }
        for (; s + 2 <= logL; s += 2) { fft_pass<4, false>(A, Bq, L, s, wt, ti, NT); __syncthreads(); }
        if (s < logL) { fft_pass<2, false>(A, Bq, L, s, wt, ti, NT); __syncthreads(); }
      } else {
        Real* xs = xsq(q);
        Real* ys = ysq(q);
        int s = 0;
        if constexpr (kF32) {
          if (tc) {
            for (; s + 4 <= logL; s += 4) {
              h16_stage(reinterpret_cast<float*>(xs), L, s, hb, ti >> 5, lane, NT / 32);
              h16_stage(reinterpret_cast<float*>(ys), L, s, hb, ti >> 5, lane, NT / 32);
              __syncthreads();
            }
          }
        }
        if (logL == 13 && P.radix == 8 && s == 0) {  // the common slab, strides fixed (FP64)
          wht_pass_fixed<8, 13, 0, NT>(xs, ti); wht_pass_fixed<8, 13, 0, NT>(ys, ti); __syncthreads();
          wht_pass_fixed<8, 13, 3, NT>(xs, ti); wht_pass_fixed<8, 13, 3, NT>(ys, ti); __syncthreads();
          wht_pass_fixed<8, 13, 6, NT>(xs, ti); wht_pass_fixed<8, 13, 6, NT>(ys, ti); __syncthreads();
          wht_pass_fixed<8, 13, 9, NT>(xs, ti); wht_pass_fixed<8, 13, 9, NT>(ys, ti); __syncthreads();
          s = 12;
        } else if (logL == 13 && s == 12) {  // after the tensor-core stages (FP32)
        } else if (P.radix == 8)
          for (; s + 3 <= logL; s += 3) { wht_pass<8>(xs, L, s, ti, NT); wht_pass<8>(ys, L, s, ti, NT); __syncthreads(); }
        for (; s + 2 <= logL; s += 2) { wht_pass<4>(xs, L, s, ti, NT); wht_pass<4>(ys, L, s, ti, NT); __syncthreads(); }
        if (logL == 13 && s == 12) {
          wht_pass_fixed<2, 13, 12, NT>(xs, ti);
          wht_pass_fixed<2, 13, 12, NT>(ys, ti);
          __syncthreads();
        } else if (s < logL) { wht_pass<2>(xs, L, s, ti, NT); wht_pass<2>(ys, L, s, ti, NT); __syncthreads(); }
      }
      // ---- accumulate over the row slots: thread tid owns m = tid + j kBT
      if (fft) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int m = tid + j * kBT;
          if (m < L) {
            if constexpr (kF32) {
              // the two rows' Z^2 are summed in FP32 (one rounding, like
              // each row's own), then added to the compensated pair
              C* zp0 = bufA(0) + ph<EC>(m);
              C* zp1 = bufA(1) + ph<EC>(m);
              const C z0 = *zp0, z1 = *zp1;
              *zp0 = mk((Real)0, (Real)0);  // clear for the next rows
              *zp1 = mk((Real)0, (Real)0);
              const float re = fmaf(-z1.y, z1.y, fmaf(z1.x, z1.x, fmaf(-z0.y, z0.y, z0.x * z0.x)));
              const float im = fmaf(z1.x, z1.y, z0.x * z0.y);
              tsum(acc[2 * j], lo[2 * j], re);
              tsum(acc[2 * j + 1], lo[2 * j + 1], im + im);
            } else {
#pragma unroll
              for (int qq = 0; qq < KB; ++qq) {
                C* zp = bufA(qq) + ph<EC>(m);
                const C z = *zp;
                *zp = mk((Real)0, (Real)0);  // clear for the next row
                acc[2 * j] = fma(z.x, z.x, fma(-z.y, z.y, acc[2 * j]));
                acc[2 * j + 1] = fma(z.x + z.x, z.y, acc[2 * j + 1]);
              }
            }
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int m = tid + j * kBT;
          if (m < L) {
            if constexpr (kF32) {  // the two rows summed in FP32 first, as for the FFT
              Real* xp0 = xsq(0) + ph<ER>(m);
              Real* yp0 = ysq(0) + ph<ER>(m);
              Real* xp1 = xsq(1) + ph<ER>(m);
              Real* yp1 = ysq(1) + ph<ER>(m);
              const float sxy = fmaf(*xp1, *yp1, *xp0 * *yp0);
              *xp0 = 0.f;  // clear for the next rows
              *yp0 = 0.f;
              *xp1 = 0.f;
              *yp1 = 0.f;
              tsum(acc[j], lo[j], sxy);
            } else {
#pragma unroll
              for (int qq = 0; qq < KB; ++qq) {
                Real* xp = xsq(qq) + ph<ER>(m);
                Real* yp = ysq(qq) + ph<ER>(m);
                const Real xv = *xp, yv = *yp;
                *xp = (Real)0;  // clear for the next row
                *yp = (Real)0;
                acc[j] = fma(xv, yv, acc[j]);
              }
            }
          }
        }
      }
      __syncthreads();  // the slots are read before the next rows clear them
    }
    if (fft) {
      double2* out = reinterpret_cast<double2*>(P.partial) +
                     (((size_t)I.g * P.d + I.t) * (size_t)R + I.r) * (size_t)L;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int m = tid + j * kBT;
        if (m < L)
          out[m] = make_double2((double)acc[2 * j] + (double)lo[2 * j], (double)acc[2 * j + 1] + (double)lo[2 * j + 1]);
      }
    } else {
      double* out = reinterpret_cast<double*>(P.partial) +
                    (((size_t)I.g * P.d + I.t) * (size_t)R + I.r) * (size_t)L;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int m = tid + j * kBT;
        if (m < L) out[m] = (double)acc[j] + (double)lo[j];
      }
    }
  }
}

// ---------------------------------------------------------- batched finalize
// One CTA per (product, repetition t) with b <= 2^14: the k-group reduction
// of the slab partials and the inverse transform in shared memory, in FP64.
// FFT: P[f] = (Q[f] - conj(Q[-f])) / (4i) is the spectrum of the real p;
// p is recovered from a half-length complex inverse of
//   Z[k] = (P[k] + P[k + b/2]) + i (P[k] - P[k + b/2]) w_b^{-k},  k < b/2,
// whose output is z[n] = b (p[2n] + i p[2n+1]).  FWHT: p = WHT_b(P) / b.
constexpr int kFinThreads = 1024;

__global__ void __launch_bounds__(kFinThreads, 1) k_finalize_jobs(const FinJob* __restrict__ jobs) {
  const FinJob J = jobs[blockIdx.x];
  extern __shared__ __align__(16) unsigned char sfin[];
  const int tid = threadIdx.x;
  const int b = 1 << J.log2b, L = 1 << J.logL, logR = J.log2b - J.logL, R = 1 << logR;
  if (J.variant == kVariantFFT) {
    const double2* part = reinterpret_cast<const double2*>(J.partial);
    const size_t gstride = (size_t)J.d * (size_t)b;
    const size_t tbase = (size_t)J.t * (size_t)b;
    auto Q = [&](int f) {  // sum over k-groups at frequency f = R m + r
      const size_t off = tbase + ((size_t)(f & (R - 1)) << J.logL) + (size_t)(f >> logR);
      double2 q = make_double2(0.0, 0.0);
      for (int g = 0; g < J.G; ++g) {
        const double2 v = part[(size_t)g * gstride + off];
        q.x += v.x;
        q.y += v.y;
      }
      return q;
    };
    auto P = [&](int f) {
      const double2 q = Q(f), qn = Q((b - f) & (b - 1));
      return make_double2(0.25 * (q.y + qn.y), -0.25 * (q.x - qn.x));
    };
    const int logM = J.log2b - 1, M = 1 << logM;
    double2* z = reinterpret_cast<double2*>(sfin);
    for (int k = tid; k < M; k += kFinThreads) {
      const double2 x0 = P(k), x1 = P(k + M);
      const double2 w = J.tw[k];  // w_b^k; the conjugate is used
      const double dx = x0.x - x1.x, dy = x0.y - x1.y;
      const double ex = dx * w.x + dy * w.y, ey = dy * w.x - dx * w.y;  // (x0 - x1) conj(w)
      z[ph<16>((int)brev_bits((uint32_t)k, logM))] = make_double2(x0.x + x1.x - ey, x0.y + x1.y + ex);
    }
    __syncthreads();
    for (int st = 0; st < logM; ++st) {  // inverse DIT, conjugate twiddles
      const int half = 1 << st;
      for (int p = tid; p < (M >> 1); p += kFinThreads) {
        const int kk = p & (half - 1);
        const int ia = ((p >> st) << (st + 1)) | kk, ic = ia + half;
        const double2 w = J.tw[(size_t)kk << (J.log2b - st - 1)];
        const double2 u = z[ph<16>(ia)], v = z[ph<16>(ic)];
        const double2 vw = make_double2(v.x * w.x + v.y * w.y, v.y * w.x - v.x * w.y);
        z[ph<16>(ia)] = make_double2(u.x + vw.x, u.y + vw.y);
        z[ph<16>(ic)] = make_double2(u.x - vw.x, u.y - vw.y);
      }
      __syncthreads();
    }
    const double inv = 1.0 / (double)b;
    for (int n = tid; n < M; n += kFinThreads) {
      const double2 v = z[ph<16>(n)];
      J.p[(size_t)J.t * b + 2 * n] = v.x * inv;
      J.p[(size_t)J.t * b + 2 * n + 1] = v.y * inv;
    }
  } else {
    const double* part = reinterpret_cast<const double*>(J.partial);
    const size_t gstride = (size_t)J.d * (size_t)b;
    double* x = reinterpret_cast<double*>(sfin);
    for (int f = tid; f < b; f += kFinThreads) {  // f = r L + m is the slab layout itself
      double q = 0.0;
      for (int g = 0; g < J.G; ++g) q += part[(size_t)g * gstride + (size_t)J.t * b + f];
      x[ph<8>(f)] = q;
    }
    __syncthreads();
    for (int st = 0; st < J.log2b; ++st) {
      const int half = 1 << st;
      for (int p = tid; p < (b >> 1); p += kFinThreads) {
        const int ia = ((p >> st) << (st + 1)) | (p & (half - 1)), ic = ia + half;
        const double u = x[ph<8>(ia)], v = x[ph<8>(ic)];
        x[ph<8>(ia)] = u + v;
        x[ph<8>(ic)] = u - v;
      }
      __syncthreads();
    }
    const double inv = 1.0 / (double)b;
    for (int f = tid; f < b; f += kFinThreads) J.p[(size_t)J.t * b + f] = x[ph<8>(f)] * inv;
  }
  (void)L;
}

bool batch_finalize_fits(int log2b) { return log2b >= 2 && log2b <= 14; }

void batch_launch_finalize(const FinJob* dJobs, int n_jobs, cudaStream_t s) {
  if (n_jobs <= 0) return;
  const size_t smem = 147456;  // 2^13 complex FP64 (or 2^14 real) + padding
  CMM_CUDA(cudaFuncSetAttribute(k_finalize_jobs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ProfScope prof("finalize", s);
  count_launch();
  k_finalize_jobs<<<(unsigned)n_jobs, kFinThreads, smem, s>>>(dJobs);
  CMM_CUDA(cudaGetLastError());
}

// per-k exponent balance of many products (FFT): the same rule as the
// single-product kernels (k_row_scale / k_row_scale_f32)
struct ScaleJob {
  const void* AT;
  const void* B;
  int* out;
  int64_t n_a, n_inner, n_b;
};

template <typename Real>
__global__ void k_row_scale_jobs(const ScaleJob* __restrict__ jobs) {
  const ScaleJob J = jobs[blockIdx.y];
  __shared__ double sa[32], sb[32];
  for (int64_t k = blockIdx.x; k < J.n_inner; k += gridDim.x) {
    const Real* ra = reinterpret_cast<const Real*>(J.AT) + (size_t)k * (size_t)J.n_a;
    const Real* rb = reinterpret_cast<const Real*>(J.B) + (size_t)k * (size_t)J.n_b;
    double ma = 0.0, mb = 0.0;
    for (int64_t i = threadIdx.x; i < J.n_a; i += blockDim.x) ma = fmax(ma, fabs((double)__ldg(ra + i)));
    for (int64_t j = threadIdx.x; j < J.n_b; j += blockDim.x) mb = fmax(mb, fabs((double)__ldg(rb + j)));
    for (int o = 16; o > 0; o >>= 1) {
      ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
      mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sa[w] = ma; sb[w] = mb; }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int i = 1; i < (int)(blockDim.x >> 5); ++i) { ma = fmax(ma, sa[i]); mb = fmax(mb, sb[i]); }
      int e;
      if (!(ma > 0.0) || !(mb > 0.0)) {
        e = (ma == 0.0 || mb == 0.0) ? kBSkip : 0;
      } else {
        auto ex = [](double m) { return (int)((__double_as_longlong(m) >> 52) & 0x7ff) - 1023; };
        const int lim = sizeof(Real) == 4 ? 60 : 400;
        e = (ex(ma) - ex(mb)) / 2;
        e = e > lim ? lim : (e < -lim ? -lim : e);
      }
      J.out[k] = e;
    }
    __syncthreads();
  }
}

// ================================================================== host

namespace {

struct TuneKey {
  int variant, f32, log2b, nlog;
  bool operator<(const TuneKey& o) const {
    return std::tie(variant, f32, log2b, nlog) < std::tie(o.variant, o.f32, o.log2b, o.nlog);
  }
};
struct TuneVal {
  int logL, radix, tc;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;  // process-wide autotuner cache

int ilog2c(int64_t x) {
  int l = 0;
  while (((int64_t)1 << l) < x) ++l;
  return l;
}

size_t smem_bytes(bool f32) {
  const size_t real = f32 ? 4 : 8, cpx = 2 * real;
  const size_t L = (size_t)1 << kBFftLog, W = (size_t)1 << kBWhtLog;
  const size_t plf = f32 ? L + L / 16 : L + L / 8, plw = f32 ? W + W / 32 : W + W / 16;
  const size_t per_row = std::max(2 * plf * cpx, 2 * plw * real);
  return (f32 ? 2 : 1) * per_row + (L + 256 + 256) * cpx;
}

template <typename Real>
void launch_sketch(const BProd* dP, const BItem* dI, int n_items, int* dCounter, const double2* tw4096,
                   int ctas, cudaStream_t s) {
  const size_t smem = smem_bytes(sizeof(Real) == 4);
  CMM_CUDA(cudaFuncSetAttribute(k_batch_sketch<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CMM_CUDA(cudaMemsetAsync(dCounter, 0, sizeof(int), s));
  ProfScope prof("sketch", s);
  count_launch();
  k_batch_sketch<Real><<<ctas, kBT, smem, s>>>(dP, dI, n_items, dCounter, tw4096);
  CMM_CUDA(cudaGetLastError());
}

template <typename Real>
int resident_ctas() {
  int per_sm = 0;
  CMM_CUDA(cudaFuncSetAttribute(k_batch_sketch<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem_bytes(sizeof(Real) == 4)));
  CMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_sketch<Real>, kBT,
                                                         smem_bytes(sizeof(Real) == 4)));
  if (per_sm < 1) throw unsupported("batch sketch kernel does not fit an SM");
  return per_sm * num_sms();
}

}  // namespace

int batch_resident_ctas(bool f32) { return f32 ? resident_ctas<float>() : resident_ctas<double>(); }

void batch_launch_sketch(bool f32, const BProd* dP, const BItem* dI, int n_items, int* dCounter,
                         const double2* tw4096, int ctas, cudaStream_t s) {
  if (n_items <= 0) return;
  if (f32) launch_sketch<float>(dP, dI, n_items, dCounter, tw4096, ctas, s);
  else launch_sketch<double>(dP, dI, n_items, dCounter, tw4096, ctas, s);
}

bool batch_tuned(int variant, bool f32, int log2b, int64_t n_ab, int* logL, int* radix, int* tc) {
  const TuneKey key{variant, (int)f32, log2b, ilog2c(std::max<int64_t>(n_ab, 1))};
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto it = g_tune.find(key);
  if (it == g_tune.end()) return false;
  *logL = it->second.logL;
  *radix = it->second.radix;
  *tc = it->second.tc;
  return true;
}

double batch_unit_cost(int64_t n_a, int64_t n_b, int logL) {
  return 4.0 * (double)(n_a + n_b) + (double)(1 << logL) * (double)std::max(logL, 1);
}

struct BatchPlan {
  bool f32 = false;
  int count = 0;
  std::vector<cmm_batch_product> prods;
  std::vector<SketchPlan> plans;  // slab geometry + k-groups per product (finalize)
  std::vector<SlabPlan> splans;   // per product: indices sorted by slab position
  std::vector<int> radix, tuned, tc;
  std::vector<const double2*> tw;  // w_b table per product
  std::vector<size_t> off_codesA, off_codesB, off_scale, off_partial;
  cudaStream_t stream = nullptr;  // creation stream (owns the buffers)
  DevBuf params, codes, scale, partial, work, dprods, ditems, counter, hjobs, sjobs, fjobs;
  int n_fjobs = 0;  // batched finalize jobs (b <= 2^14); other products finalize one by one
  int n_items = 0, ctas = 0, n_scale_jobs = 0;
  int64_t max_hash_total = 0, max_inner = 0;
  const double2* tw4096 = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t launches_per_run = 0;
  ~BatchPlan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

namespace {

// sorted plan of product i for slab length 2^logL (R2 = 1: one segment per t)
SlabPlan make_sorted(const BatchPlan& B, int i, int logL, cudaStream_t s) {
  const cmm_batch_product& q = B.prods[(size_t)i];
  return make_residue_plan(B.codes.as<uint32_t>() + B.off_codesA[(size_t)i],
                           B.codes.as<uint32_t>() + B.off_codesB[(size_t)i], q.n_a, q.n_b, q.d, q.b, logL, 0, s);
}

// host copy of the device description of product i
BProd make_bprod(const BatchPlan& B, int i, void* partial, const SlabPlan& sp) {
  const cmm_batch_product& q = B.prods[(size_t)i];
  const SketchPlan& P = B.plans[(size_t)i];
  BProd d{};
  d.AT = q.AT;
  d.B = q.B;
  d.srcA = sp.srcA.as<uint32_t>();
  d.srcB = sp.srcB.as<uint32_t>();
  d.codeA = sp.codeA.ptr;
  d.codeB = sp.codeB.ptr;
  d.cutA = sp.countA.as<uint32_t>();
  d.cutB = sp.countB.as<uint32_t>();
  d.SA = sp.EA;
  d.SB = sp.EB;
  d.code16 = sp.u16 ? 1 : 0;
  d.scale = B.scale.as<int>() + B.off_scale[(size_t)i];
  d.tw = B.tw[(size_t)i];
  d.partial = partial;
  d.n_a = q.n_a;
  d.n_inner = q.n_inner;
  d.n_b = q.n_b;
  d.d = q.d;
  d.log2b = P.log2b;
  d.logL = P.logL;
  d.logR = P.logR;
  d.G = P.G;
  d.variant = q.variant;
  d.radix = B.radix[(size_t)i];
  d.tc = B.tc[(size_t)i];
  return d;
}

void set_geometry(SketchPlan& P, int logL) {
  P.logL = logL;
  P.L = 1 << logL;
  P.logR = P.log2b - logL;
  P.R = 1 << P.logR;
  P.KB = 1;
}

// relative cost of one (t, slab, k) unit: scatter of n_a + n_b elements
// plus an L-point transform
double unit_cost(const cmm_batch_product& q, int logL) {
  return 4.0 * (double)(q.n_a + q.n_b) + (double)(1 << logL) * (double)std::max(logL, 1);
}

// row exponents of the FFT products (the first graph node: they depend on
// the inputs' contents)
void enqueue_scale(BatchPlan& B, cudaStream_t s) {
  if (B.n_scale_jobs) {
    const int64_t bx = std::min<int64_t>(std::max<int64_t>(B.max_inner, 1), 2048);
    ProfScope prof("scale", s);
    count_launch();
    if (B.f32)
      k_row_scale_jobs<float><<<dim3((unsigned)bx, (unsigned)B.n_scale_jobs), 256, 0, s>>>(B.sjobs.as<ScaleJob>());
    else
      k_row_scale_jobs<double><<<dim3((unsigned)bx, (unsigned)B.n_scale_jobs), 256, 0, s>>>(B.sjobs.as<ScaleJob>());
    CMM_CUDA(cudaGetLastError());
  }
}

void enqueue(BatchPlan& B, cudaStream_t s) {
  enqueue_scale(B, s);
  if (B.n_items > 0) {
    if (B.f32)
      launch_sketch<float>(B.dprods.as<BProd>(), B.ditems.as<BItem>(), B.n_items, B.counter.as<int>(),
                           B.tw4096, B.ctas, s);
    else
      launch_sketch<double>(B.dprods.as<BProd>(), B.ditems.as<BItem>(), B.n_items, B.counter.as<int>(),
                            B.tw4096, B.ctas, s);
  }
  batch_launch_finalize(B.fjobs.as<FinJob>(), B.n_fjobs, s);
  for (int i = 0; i < B.count; ++i) {
    const cmm_batch_product& q = B.prods[(size_t)i];
    if (!batch_finalize_fits(B.plans[(size_t)i].log2b))
      launch_finalize(B.plans[(size_t)i], B.partial.as<unsigned char>() + B.off_partial[(size_t)i], B.tw[(size_t)i],
                      B.work.ptr, q.p, s);
    if (q.C)
      launch_decompress_dense(q.variant, q.d, q.b, q.n_a, q.n_b, B.codes.as<uint32_t>() + B.off_codesA[(size_t)i],
                              B.codes.as<uint32_t>() + B.off_codesB[(size_t)i], q.p, q.C, s);
  }
}

// Times the candidate (slab length, radix) pairs of product i on its own
// data over its first rows, with enough k-groups to fill the device.
TuneVal autotune(BatchPlan& B, int i, cudaStream_t s) {
  const cmm_batch_product& q = B.prods[(size_t)i];
  const int log2b = B.plans[(size_t)i].log2b;
  const int lmax = q.variant == kVariantFFT ? kBFftLog : kBWhtLog;
  std::vector<TuneVal> cand;
  // FP32 FWHT also weighs the tensor-core Hadamard-16 stages against CUDA cores
  const bool tc_choice = B.f32 && q.variant == kVariantFWHT;
  for (int dl = 0; dl < 3; ++dl) {
    const int logL = std::min(log2b, lmax) - dl;  // slab lengths L, L/2, L/4
    if (logL < 1) continue;
    for (int rx : {8, 4}) {
      cand.push_back({logL, rx, 1});
      if (tc_choice && logL >= 8) cand.push_back({logL, rx, 0});
    }
  }
  const int64_t rows = std::min<int64_t>(q.n_inner, 96);
  float best_ms = 1e30f;
  TuneVal best = cand.front();
  cudaEvent_t e0, e1;
  CMM_CUDA(cudaEventCreate(&e0));
  CMM_CUDA(cudaEventCreate(&e1));
  DevBuf cnt(sizeof(int), s), dP(sizeof(BProd), s);
  for (const TuneVal& c : cand) {
    SketchPlan P = B.plans[(size_t)i];
    set_geometry(P, c.logL);
    const int units = P.R * q.d;
    int G = (int)std::max<int64_t>(1, std::min<int64_t>(rows, (B.ctas + units - 1) / units));
    P.G = G;
    DevBuf part((size_t)G * q.d * (size_t)q.b * (q.variant == kVariantFFT ? 16 : 8), s);
    const SlabPlan sp = make_sorted(B, i, c.logL, s);
    const SketchPlan keep = B.plans[(size_t)i];
    const int keep_rx = B.radix[(size_t)i], keep_tc = B.tc[(size_t)i];
    B.plans[(size_t)i] = P;
    B.radix[(size_t)i] = c.radix;
    B.tc[(size_t)i] = c.tc;
    BProd bp = make_bprod(B, i, part.ptr, sp);
    bp.n_inner = rows;  // the first rows only
    B.plans[(size_t)i] = keep;
    B.radix[(size_t)i] = keep_rx;
    B.tc[(size_t)i] = keep_tc;
    std::vector<BItem> its;
    for (int g = 0; g < G; ++g)
      for (int t = 0; t < q.d; ++t)
        for (int r = 0; r < P.R; ++r) its.push_back({0, t, r, g});
    DevBuf dI(its.size() * sizeof(BItem), s);
    CMM_CUDA(cudaMemcpyAsync(dP.ptr, &bp, sizeof(BProd), cudaMemcpyHostToDevice, s));
    CMM_CUDA(cudaMemcpyAsync(dI.ptr, its.data(), its.size() * sizeof(BItem), cudaMemcpyHostToDevice, s));
    const int ctas = std::min<int>(B.ctas, (int)its.size());
    float ms = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      CMM_CUDA(cudaEventRecord(e0, s));
      if (B.f32) launch_sketch<float>(dP.as<BProd>(), dI.as<BItem>(), (int)its.size(), cnt.as<int>(), B.tw4096, ctas, s);
      else launch_sketch<double>(dP.as<BProd>(), dI.as<BItem>(), (int)its.size(), cnt.as<int>(), B.tw4096, ctas, s);
      CMM_CUDA(cudaEventRecord(e1, s));
      CMM_CUDA(cudaEventSynchronize(e1));
      float t = 0.f;
      CMM_CUDA(cudaEventElapsedTime(&t, e0, e1));
      if (rep > 0) ms = std::min(ms, t);  // the first launch warms up
    }
    if (getenv("CMM_DEBUG"))
      fprintf(stderr, "[cmm] batch tune candidate: variant=%d b=%d L=%d radix=%d tc=%d: %.3f ms\n", q.variant, q.b,
              1 << c.logL, c.radix, c.tc, ms);
    if (ms < best_ms) { best_ms = ms; best = c; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (getenv("CMM_DEBUG"))
    fprintf(stderr, "[cmm] batch tune: variant=%d f32=%d b=%d n=%lld -> L=%d radix=%d tc=%d (%.3f ms)\n",
            q.variant, (int)B.f32, q.b, (long long)(q.n_a + q.n_b), 1 << best.logL, best.radix, best.tc, best_ms);
  return best;
}

}  // namespace

BatchPlan* batch_create(const cmm_batch_product* products, int count, bool f32, bool tune) {
  if (count < 0) throw invalid_argument("count must not be negative");
  if (count > 0 && !products) throw invalid_argument("products must not be null");
  // argument checks first (no CUDA call before all products are valid)
  for (int i = 0; i < count; ++i) {
    const cmm_batch_product& q = products[i];
    const std::string who = "product " + std::to_string(i) + ": ";
    if (q.variant != kVariantFFT && q.variant != kVariantFWHT) throw invalid_argument(who + "invalid variant");
    if (q.b < 2 || (q.b & (q.b - 1)) != 0)
      throw invalid_argument(who + "b must be power of 2 greater than 1 (got " + std::to_string(q.b) + ")");
    if (q.d < 1) throw invalid_argument(who + "d must be positive (got " + std::to_string(q.d) + ")");
    if (q.hash_kind < 0 || q.hash_kind > 3)
      throw invalid_argument(who +
                             "Invalid hash provided; hash must be one of `multiply shift', `multiply add "
                             "shift', `tabulation8', or `tabulation16'");
    if (ilog2c(q.b) > kMaxLog2B) throw unsupported(who + "b exceeds the largest supported b (2^24)");
    if (q.d > 65535) throw unsupported(who + "d > 65535 is not supported");
    if (q.n_a < 0 || q.n_inner < 0 || q.n_b < 0) throw invalid_argument(who + "negative matrix dimension");
    if (q.n_a > 4294967296LL || q.n_b > 4294967296LL) throw unsupported(who + "dimension above 2^32");
    if (q.n_inner > 0 && q.n_a > 0 && !q.AT) throw invalid_argument(who + "AT is null");
    if (q.n_inner > 0 && q.n_b > 0 && !q.B) throw invalid_argument(who + "B is null");
    if (!q.p) throw invalid_argument(who + "p is null");
  }
  std::unique_ptr<BatchPlan> B(new BatchPlan());
  B->f32 = f32;
  B->count = count;
  B->prods.assign(products, products + count);
  CMM_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
  cudaStream_t s = B->stream;
  B->ctas = f32 ? resident_ctas<float>() : resident_ctas<double>();
  B->tw4096 = twiddles(1 << kBFftLog, s);

  // ---- validation, hash parameters, buffer offsets
  std::vector<uint8_t> blob;
  std::vector<size_t> off_params((size_t)count), fn_bytes((size_t)count);
  size_t ncodes = 0, nscale = 0;
  B->plans.resize((size_t)count);
  B->radix.assign((size_t)count, 8);
  B->tc.assign((size_t)count, 1);
  B->tuned.assign((size_t)count, 0);
  B->tw.resize((size_t)count);
  B->off_codesA.resize((size_t)count);
  B->off_codesB.resize((size_t)count);
  B->off_scale.resize((size_t)count);
  B->off_partial.resize((size_t)count);
  for (int i = 0; i < count; ++i) {
    const cmm_batch_product& q = B->prods[(size_t)i];
    const SketchParams sp = make_sketch_params(q.hash_kind, q.d, q.b, q.seed);
    off_params[(size_t)i] = blob.size();
    fn_bytes[(size_t)i] = sp.fn_bytes;
    blob.insert(blob.end(), sp.blob.begin(), sp.blob.end());
    while (blob.size() % 16) blob.push_back(0);
    SketchPlan& P = B->plans[(size_t)i];
    P = SketchPlan{};
    P.variant = q.variant;
    P.d = q.d;
    P.b = q.b;
    P.log2b = ilog2c(q.b);
    P.n_a = q.n_a;
    P.n_inner = q.n_inner;
    P.n_b = q.n_b;
    set_geometry(P, std::min(P.log2b, q.variant == kVariantFFT ? kBFftLog : kBWhtLog));
    P.G = 1;
    B->tw[(size_t)i] = twiddles(q.b, s);
    B->off_codesA[(size_t)i] = ncodes;
    ncodes += (size_t)q.d * (size_t)q.n_a;
    B->off_codesB[(size_t)i] = ncodes;
    ncodes += (size_t)q.d * (size_t)q.n_b;
    ncodes = (ncodes + 63) & ~(size_t)63;
    B->off_scale[(size_t)i] = nscale;
    nscale += (size_t)std::max<int64_t>(q.n_inner, 1);
    B->max_hash_total = std::max(B->max_hash_total, (int64_t)q.d * std::max(q.n_a, q.n_b));
    B->max_inner = std::max(B->max_inner, q.n_inner);
  }
  B->params = DevBuf(std::max<size_t>(blob.size(), 16), s);
  if (!blob.empty()) CMM_CUDA(cudaMemcpyAsync(B->params.ptr, blob.data(), blob.size(), cudaMemcpyHostToDevice, s));
  B->codes = DevBuf(std::max<size_t>(ncodes, 1) * 4, s);
  B->scale = DevBuf(std::max<size_t>(nscale, 1) * 4, s);

  // ---- hash / scale job tables
  std::vector<HashJob> hj;
  std::vector<ScaleJob> sj;
  for (int i = 0; i < count; ++i) {
    const cmm_batch_product& q = B->prods[(size_t)i];
    const uint8_t* base = B->params.as<uint8_t>() + off_params[(size_t)i];
    const size_t set = fn_bytes[(size_t)i] * (size_t)q.d;
    const int log2b = B->plans[(size_t)i].log2b;
    hj.push_back({base, base + 2 * set, B->codes.as<uint32_t>() + B->off_codesA[(size_t)i], q.n_a, q.d, log2b, q.hash_kind});
    hj.push_back({base + set, base + 3 * set, B->codes.as<uint32_t>() + B->off_codesB[(size_t)i], q.n_b, q.d, log2b, q.hash_kind});
    if (q.variant == kVariantFFT && q.n_inner > 0)
      sj.push_back({q.AT, q.B, B->scale.as<int>() + B->off_scale[(size_t)i], q.n_a, q.n_inner, q.n_b});
  }
  B->n_scale_jobs = (int)sj.size();
  B->hjobs = DevBuf(std::max<size_t>(hj.size(), 1) * sizeof(HashJob), s);
  B->sjobs = DevBuf(std::max<size_t>(sj.size(), 1) * sizeof(ScaleJob), s);
  if (!hj.empty()) CMM_CUDA(cudaMemcpyAsync(B->hjobs.ptr, hj.data(), hj.size() * sizeof(HashJob), cudaMemcpyHostToDevice, s));
  if (!sj.empty()) CMM_CUDA(cudaMemcpyAsync(B->sjobs.ptr, sj.data(), sj.size() * sizeof(ScaleJob), cudaMemcpyHostToDevice, s));
  B->counter = DevBuf(sizeof(int), s);

  // ---- hash codes (fixed by the plan's seeds and sizes) and the current
  // row exponents, which the sorted plans and the autotuner read
  launch_hash_codes_jobs(B->hjobs.as<HashJob>(), 2 * count, B->max_hash_total, s);
  enqueue_scale(*B, s);

  // ---- per-class configuration (autotuned, cached)
  for (int i = 0; i < count; ++i) {
    const cmm_batch_product& q = B->prods[(size_t)i];
    SketchPlan& P = B->plans[(size_t)i];
    const TuneKey key{q.variant, (int)f32, P.log2b, ilog2c(std::max<int64_t>(q.n_a + q.n_b, 1))};
    TuneVal v{P.logL, 8, 1};
    bool have = false;
    {
      std::lock_guard<std::mutex> g(g_tune_mu);
      auto it = g_tune.find(key);
      if (it != g_tune.end()) { v = it->second; have = true; }
    }
    if (!have && tune && q.n_inner > 0) {
      v = autotune(*B, i, s);
      std::lock_guard<std::mutex> g(g_tune_mu);
      g_tune[key] = v;
      have = true;
    }
    set_geometry(P, v.logL);
    B->radix[(size_t)i] = v.radix;
    B->tc[(size_t)i] = v.tc;
    B->tuned[(size_t)i] = have ? 1 : 0;
  }

  // ---- k-groups: items of about equal cost, several per resident CTA
  double total = 0.0;
  for (int i = 0; i < count; ++i) {
    const cmm_batch_product& q = B->prods[(size_t)i];
    const SketchPlan& P = B->plans[(size_t)i];
    total += (double)q.n_inner * P.R * q.d * unit_cost(q, P.logL);
  }
  const double target = std::max(total / ((double)B->ctas * 6.0), 1.0);
  size_t npart = 0;
  struct Cost { double c; BItem it; };
  std::vector<Cost> items;
  for (int i = 0; i < count; ++i) {
    const cmm_batch_product& q = B->prods[(size_t)i];
    SketchPlan& P = B->plans[(size_t)i];
    const double row = unit_cost(q, P.logL);
    int64_t G = (int64_t)std::ceil((double)q.n_inner * row / target);
    const int64_t gmin = std::max<int64_t>(1, q.n_inner / 8);  // at least 8 rows per item
    G = std::max<int64_t>(1, std::min<int64_t>({G, gmin, 65535}));
    P.G = (int)G;
    B->off_partial[(size_t)i] = npart;
    npart += (size_t)P.G * q.d * (size_t)q.b * (q.variant == kVariantFFT ? 16 : 8);
    npart = (npart + 255) & ~(size_t)255;
    if (q.n_inner == 0) continue;  // finalize alone writes p = 0
    const int64_t per = (q.n_inner + G - 1) / G;
    for (int64_t g = 0; g < G; ++g) {
      const int64_t rows = std::min<int64_t>(per, q.n_inner - g * per);
      if (rows <= 0) continue;
      for (int t = 0; t < q.d; ++t)
        for (int r = 0; r < P.R; ++r) items.push_back({(double)rows * row, {i, t, r, (int)g}});
    }
  }
  // longest first; k-groups without rows still need zero partials
  std::stable_sort(items.begin(), items.end(), [](const Cost& a, const Cost& b) { return a.c > b.c; });
  if (items.size() > (size_t)2147483647) throw unsupported("too many batch work items");
  B->n_items = (int)items.size();
  B->partial = DevBuf(std::max<size_t>(npart, 256), s);
  CMM_CUDA(cudaMemsetAsync(B->partial.ptr, 0, std::max<size_t>(npart, 256), s));
  size_t work = 16;
  for (int i = 0; i < count; ++i) work = std::max(work, 2 * (size_t)B->prods[(size_t)i].d * (size_t)B->prods[(size_t)i].b * 16);
  B->work = DevBuf(work, s);
  std::vector<BProd> bp;
  B->splans.resize((size_t)count);
  for (int i = 0; i < count; ++i) {
    B->splans[(size_t)i] = make_sorted(*B, i, B->plans[(size_t)i].logL, s);
    bp.push_back(make_bprod(*B, i, B->partial.as<unsigned char>() + B->off_partial[(size_t)i], B->splans[(size_t)i]));
  }
  std::vector<BItem> bi;
  for (const Cost& c : items) bi.push_back(c.it);
  std::vector<FinJob> fj;
  for (int i = 0; i < count; ++i) {
    const SketchPlan& P = B->plans[(size_t)i];
    if (!batch_finalize_fits(P.log2b)) continue;
    for (int t = 0; t < P.d; ++t)
      fj.push_back({B->partial.as<unsigned char>() + B->off_partial[(size_t)i], B->prods[(size_t)i].p, B->tw[(size_t)i],
                    P.G, P.d, t, P.log2b, P.logL, P.variant});
  }
  B->n_fjobs = (int)fj.size();
  B->fjobs = DevBuf(std::max<size_t>(fj.size(), 1) * sizeof(FinJob), s);
  if (!fj.empty()) CMM_CUDA(cudaMemcpyAsync(B->fjobs.ptr, fj.data(), fj.size() * sizeof(FinJob), cudaMemcpyHostToDevice, s));
  B->dprods = DevBuf(std::max<size_t>(bp.size(), 1) * sizeof(BProd), s);
  B->ditems = DevBuf(std::max<size_t>(bi.size(), 1) * sizeof(BItem), s);
  if (!bp.empty()) CMM_CUDA(cudaMemcpyAsync(B->dprods.ptr, bp.data(), bp.size() * sizeof(BProd), cudaMemcpyHostToDevice, s));
  if (!bi.empty()) CMM_CUDA(cudaMemcpyAsync(B->ditems.ptr, bi.data(), bi.size() * sizeof(BItem), cudaMemcpyHostToDevice, s));
  B->ctas = std::max(1, std::min(B->ctas, B->n_items));
  CMM_CUDA(cudaStreamSynchronize(s));
  return B.release();
}

void batch_run(BatchPlan* B, cudaStream_t user) {
  if (!B) throw invalid_argument("batch handle is null");
  cudaStream_t s = user ? user : B->stream;
  if (!B->exec) {
    // capture once: the sequence depends only on the plan
    const bool prev = prof_set(false);
    const int64_t before = cmm_launch_count();
    cudaStream_t cs = B->stream;  // capture on the plan's own stream
    CMM_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed));
    try {
      enqueue(*B, cs);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(cs, &g);
      if (g) cudaGraphDestroy(g);
      prof_set(prev);
      throw;
    }
    CMM_CUDA(cudaStreamEndCapture(cs, &B->graph));
    CMM_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
    prof_set(prev);
    B->launches_per_run = cmm_launch_count() - before;
    count_launch(-(int)B->launches_per_run);  // captured, not launched
  }
  {
    ProfScope prof("batch", s);
    CMM_CUDA(cudaGraphLaunch(B->exec, s));
  }
  count_launch((int)B->launches_per_run);
  if (!user) CMM_CUDA(cudaStreamSynchronize(s));
}

void batch_info(const BatchPlan* B, int64_t* items, int* ctas, int* launches) {
  if (!B) throw invalid_argument("batch handle is null");
  if (items) *items = B->n_items;
  if (ctas) *ctas = B->ctas;
  if (launches) {
    // kernels per run: scale (if any), sketch (if any), the batched finalize,
    // 3 per other finalize, 1 per dense C
    int n = (B->n_scale_jobs ? 1 : 0) + (B->n_items ? 1 : 0) + (B->n_fjobs ? 1 : 0);
    for (size_t i = 0; i < B->prods.size(); ++i) {
      const auto& q = B->prods[i];
      n += (batch_finalize_fits(B->plans[i].log2b) ? 0 : 3) + (q.C && q.n_a > 0 && q.n_b > 0 ? 1 : 0);
    }
    *launches = n;
  }
}

void batch_config(const BatchPlan* B, int i, int* log2_slab, int* radix, int* groups, int* tuned) {
  if (!B) throw invalid_argument("batch handle is null");
  if (i < 0 || i >= B->count) throw invalid_argument("product index out of range");
  if (log2_slab) *log2_slab = B->plans[(size_t)i].logL;
  if (radix) *radix = B->radix[(size_t)i];
  if (groups) *groups = B->plans[(size_t)i].G;
  if (tuned) *tuned = B->tuned[(size_t)i];
}

void batch_destroy(BatchPlan* B) {
  if (!B) return;
  cudaStream_t s = B->stream;
  if (s) cudaStreamSynchronize(s);
  delete B;  // buffers are released on s
  if (s) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
}

}  // namespace cmm
