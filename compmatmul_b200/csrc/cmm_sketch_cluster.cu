// Cluster sketch kernels: the hot path for large b.
//
// With b = R1 * R2 * L:
//  * a radix-R1 decimation in frequency splits the b frequencies into R1
//    interleaved slabs (f = R1 f' + r1 for the FFT; f = r1 (b / R1) + f' for
//    the FWHT); each slab is a length M = b / R1 transform of
//      u_r1[n1] = tw(n1, r1) * sum_q1 w(q1, r1) x[q1 M + n1];
//  * a group of R2 CTAs computes one slab by decimation in time: CTA r2
//    takes the members of residue class n1 mod R2 only (the bucket-sorted
//    plan hands each CTA its own segment of every row, so an index is
//    scattered by R1 CTAs instead of by every slab), sums them into its
//    length-L sub-sequence and transforms it in shared memory;
//  * the R2 sub-spectra are combined by a radix-R2 DFT/WHT across the
//    group: the last radix pass writes each CTA's sub-spectrum to an
//    exchange area in global memory, which stays in L2 (R2 x L elements per
//    group, four slots in rotation), and after the group barrier CTA r2 reads the
//    R2 values of its L / R2 sub-spectrum positions back and accumulates
//    Z^2 (FFT, z = alpha x + i beta y) or X * Y (FWHT) for them over k.
//    Thread-block clusters exchanging through distributed shared memory were
//    the earlier form: clusters of 8 fit 15 times on the 148 SMs, and the
//    remote reads ran at about a third of their port's peak.
//  The grid is one cooperative launch of every resident CTA, in groups of
//  R2; a group barrier is a counter in global memory.  It is split: a CTA
//  arrives for index k after its exchange write and the next row's scatter,
//  and waits for k one iteration later, after the transform of k + 1 and
//  the scatter of k + 2, so the combine of k runs behind the transform of
//  k + 1; the row after that is staged with cp.async meanwhile.  Every CTA of a group
//  runs the same k sequence (all-zero rows are skipped by all of them), so
//  all of them reach every barrier.
// Instantiations: FFT/FWHT x FP64/FP32 (FP32 = mixed precision: FP32 data,
// two-sum compensated accumulation, tensor-core Hadamard-16 stages for the
// FWHT, FP64 partials).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <stdexcept>
#include <cstdlib>

#include "cmm_fft_device.cuh"
#include "cmm_internal.h"


namespace cmm {
namespace {

constexpr int kCT = kPlanThreads;  // 512
constexpr int kCBatch = 4;  // scatter slots loaded together
constexpr int kCSkip = -0x7fffffff;

using namespace dev;

// DFT_8 with natural-order input and output
template <typename C>
__device__ __forceinline__ void dft8(C (&u)[8]) {
  C x[8] = {u[0], u[4], u[2], u[6], u[1], u[5], u[3], u[7]};
  using R = decltype(u[0].x);
  r8(x, mk((R)1, (R)0));
#pragma unroll
  for (int e = 0; e < 8; ++e) u[e] = x[e];
}

// padded shared layouts: 16- and 8-byte elements p + p/16, 4-byte p + p/32.
// One spare element per 16 keeps the radix passes conflict-free and spreads
// the scatter's bit-reversed positions (a warp's buckets differ in bits that
// land in p/16) over all banks.
template <int ES>
__device__ __forceinline__ int phys(int p) {
  return ES == 4 ? p + (p >> 5) : p + (p >> 4);
}
template <int ES>
constexpr int phys_len(int L) {
  return ES == 4 ? L + L / 32 : L + L / 16;
}

// ------------------------------------------------- tensor-core H16 (FP32)
__device__ __forceinline__ uint32_t bf16x2(float lo_e, float hi_e) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo_e)) |
         ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi_e)) << 16);
}
// x = hi + mid + lo in BF16 (8 + 8 + 8 significant bits cover FP32's 24),
// so the +-1 products on the tensor cores lose nothing before the FP32
// accumulation (a hi/lo split measured 1.02e-5 max relative error on the
// recovered values of a 16384^2, b = 2^18 product)
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
template <int STAGE>
__device__ __forceinline__ int hpt(int V, int e) {
  if (STAGE == 0) return V * 16 + e;
  if (STAGE == 1) return (V >> 4) * 256 + e * 16 + (V & 15);
  return (V >> 8) * 4096 + e * 256 + (V & 255);
}
template <int STAGE>
__device__ __forceinline__ void h16(float* buf, const uint32_t (&hb)[2][2], int warp, int lane) {
  const int gq = lane >> 2, tq = lane & 3;
  for (int tile = warp; tile < 32; tile += kCT / 32) {
    const int V0 = tile * 16;
    const int p[8] = {hpt<STAGE>(V0 + gq, 2 * tq),     hpt<STAGE>(V0 + gq, 2 * tq + 1),
                      hpt<STAGE>(V0 + gq + 8, 2 * tq), hpt<STAGE>(V0 + gq + 8, 2 * tq + 1),
                      hpt<STAGE>(V0 + gq, 2 * tq + 8), hpt<STAGE>(V0 + gq, 2 * tq + 9),
                      hpt<STAGE>(V0 + gq + 8, 2 * tq + 8), hpt<STAGE>(V0 + gq + 8, 2 * tq + 9)};
    float x[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) x[e] = buf[phys<4>(p[e])];
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
    for (int e = 0; e < 8; ++e) buf[phys<4>(p[e])] = y[e];
  }
}

}  // namespace

// Per-phase cycle counts of the cluster kernel, compiled in only with
// -DCMM_PHASE_CLOCKS (python -m compmatmul_b200.build with
// CMM_EXTRA_NVFLAGS=-DCMM_PHASE_CLOCKS): thread 0 of every CTA adds the
// clock64() time of each phase of each inner index to g_cl_phase, which
// cmm_cluster_phase_cycles() reads and clears.  Phases: 0 the local radix
// passes with the write of the sub-spectrum, 1 wait for the next staged row
// (cp.async + barrier), 2 its scatter, 3 the arrival and the group wait for
// the previous index, 4 the combine and accumulation; 5 is unused.
constexpr int kClPhases = 6;
#ifdef CMM_PHASE_CLOCKS
__device__ unsigned long long g_cl_phase[kClPhases + 1];  // + inner indices timed
#define CL_MARK(ph)                                                        \
  do {                                                                     \
    if (tid == 0) {                                                        \
      const long long now_ = clock64();                                    \
      if ((ph) >= 0) atomicAdd(&g_cl_phase[(ph)], (unsigned long long)(now_ - t_ph)); \
      t_ph = now_;                                                         \
    }                                                                      \
  } while (0)
#else
#define CL_MARK(ph) \
  do {              \
  } while (0)
#endif

struct ClArgs {
  const void* matA;  // [t][kk][R2][SA]
  const void* matB;
  const void* codeA;  // [t][R2][SA]
  const void* codeB;
  const uint32_t* countA;  // [t][R2][513] cut offsets
  const uint32_t* countB;
  const int* scale_exp;
  const double2* tw;  // w_b^j
  void* partial;      // [g][t][b] double2 (FFT) / double (FWHT)
  void* xch;          // exchange area: [group][4][R2][L] complex (FFT) / (x, y) pairs (FWHT)
  unsigned* gsync;    // arrival counters, 4 per group (one 128-byte line each), zero at launch
  int* timeout;       // host-mapped flag: a group wait ran out
  unsigned spin_limit, wait_extra;
  int tc;             // FP32 FWHT: Hadamard-16 stages on the tensor cores (else CUDA-core passes)
  int post_full;      // FFT: the post-twiddles as one table of L entries (else two factors)
  int64_t SA, SB, kc, k0;
  int d, log2b, logR1, logR2, G, accumulate;
};

// Staged slot e of a segment sits at e + e / 16 (8-byte values) or e + e / 8
// (4-byte values): neighbouring threads' ranges start a few slots apart, and
// the spare slots spread their same-index reads over the banks.
__host__ __device__ constexpr int64_t spad_len_n(int64_t n, size_t real) {
  return n + n / (real == 8 ? 16 : 8) + 1;
}
template <typename Real>
__device__ __forceinline__ int spad(int e) { return e + (e >> (sizeof(Real) == 8 ? 4 : 3)); }
template <typename Real>
__device__ __forceinline__ int64_t spad_len(int64_t n) { return spad_len_n(n, sizeof(Real)); }

// entries of the coarse DIF weight table w_b^{512 j}, j < b / 512
__host__ __device__ inline int cl_pre_hi(int log2b) { return log2b > 9 ? 1 << (log2b - 9) : 1; }

// Shared-memory layout of one CTA, shared by the kernel and the host sizing:
// the sub-spectrum buffer, then (FFT) the factored post-twiddle tables, the
// DIF weight tables when R1 > 1, the pass twiddles and w_R1; then the staged
// row values of this CTA's segments and their premixed codes.
struct ClLayout {
  size_t buf, post, pre, ptw, wr, stage, codes, total;
};
__host__ __device__ inline size_t cl_align16(size_t x) { return (x + 15) & ~(size_t)15; }
__host__ __device__ inline ClLayout cl_layout(bool fft, bool f32, bool u16, int logL, int R1, int log2b,
                                              int64_t SA, int64_t SB, bool postFull) {
  const size_t real = f32 ? 4 : 8, cpx = 2 * real;
  const size_t L = (size_t)1 << logL;
  auto plen = [](size_t n, size_t es) { return es == 4 ? n + n / 32 : n + n / 16; };
  ClLayout o;
  size_t p = 0;
  o.buf = p;
  p += fft ? plen(L, cpx) * cpx : 2 * plen(L, real) * real;
  o.post = p;
  if (fft) p += (postFull ? L : 128 + 64) * cpx;
  o.pre = p;
  if (fft && R1 > 1) p += (cl_pre_hi(log2b) + 512) * cpx;
  o.ptw = p;
  if (fft) p += (f32 ? 1176 : 592) * cpx;
  o.wr = p;
  p += 32 * real;
  o.stage = p;
  p += cl_align16((size_t)(spad_len_n(SA, real) + spad_len_n(SB, real)) * real);
  o.codes = p;
  p += cl_align16((size_t)(SA + SB) * (u16 ? 2 : 4));
  o.total = p;
  return o;
}

static __device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((uint32_t)__cvta_generic_to_shared(sdst)),
               "l"(gsrc)
               : "memory");
}
static __device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((uint32_t)__cvta_generic_to_shared(sdst)),
               "l"(gsrc)
               : "memory");
}
static __device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

static __device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
static __device__ __forceinline__ void red_release_gpu_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// VARIANT 0 = FFT, 1 = FWHT; Real = double (plain) or float (mixed); NT
// threads per CTA: 512 (one CTA per SM) or, FP64 only, 256 with half the
// sub-transform length (two CTAs per SM, whose phases overlap).
template <int VARIANT, typename Real, typename CodeT, int NT>
__global__ void __launch_bounds__(NT, kCT / NT) k_sketch_cluster(ClArgs a) {
  constexpr bool kFFT = VARIANT == kVariantFFT;
  constexpr bool kF32 = sizeof(Real) == 4;
  static_assert(NT == kCT || (NT == kCT / 2 && !kF32), "256-thread CTAs are FP64 only");
  constexpr int LOGL = ((kFFT && !kF32) ? 12 : 13) - (NT == kCT ? 0 : 1);
  constexpr int VPT = kCT / NT;  // plan ranges (of kCT per segment) per thread
  constexpr int L = 1 << LOGL;
  using C = typename std::conditional<kF32, float2, double2>::type;
  constexpr int ES = kFFT ? (int)sizeof(C) : (int)sizeof(Real);  // shared element size
  constexpr int PL = phys_len<ES>(L);
  constexpr int OUT = L / NT;  // outputs per thread (8 or 16)

  extern __shared__ __align__(16) unsigned char sm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int R1 = 1 << a.logR1, R2 = 1 << a.logR2;
  const int r2 = (int)blockIdx.x;  // this CTA's residue class; blockIdx.y is its group
  const int logM = a.log2b - a.logR1;  // M = b / R1
  const double2* tw = a.tw;

  // ---- shared layout (cl_layout)
  const bool postFull = kFFT && a.post_full;  // w_M^{n r2} tabulated for every n < L
  const ClLayout lay = cl_layout(kFFT, kF32, sizeof(CodeT) == 2, LOGL, R1, a.log2b, a.SA, a.SB, postFull);
  C* buf0 = reinterpret_cast<C*>(sm + lay.buf);        // FFT: PL complex
  Real* xs0 = reinterpret_cast<Real*>(sm + lay.buf);   // FWHT: x: PL, y: PL real
  C* postLo = reinterpret_cast<C*>(sm + lay.post);     // FFT: w_M^{n r2} = postLo[n] (full table) or
                                                       //   postHi[n >> 7] postLo[n & 127]
  C* postHi = postLo + 128;
  C* preHi = reinterpret_cast<C*>(sm + lay.pre);       // FFT, R1 > 1: w_b^{x}, x = hi * 512 + lo
  C* preLo = preHi + cl_pre_hi(a.log2b);
  C* ptw = reinterpret_cast<C*>(sm + lay.ptw);         // FFT pass twiddles (592 FP64, 1176 FP32)
  Real* wRx = reinterpret_cast<Real*>(sm + lay.wr);    // FFT: Re/Im w_R1^j, j < 16
  Real* wRy = wRx + 16;
  Real* stA = reinterpret_cast<Real*>(sm + lay.stage);  // staged row values, this CTA's segments
  Real* stB = stA + spad_len<Real>(a.SA);
  CodeT* cA = reinterpret_cast<CodeT*>(sm + lay.codes);
  CodeT* cB = cA + a.SA;

  // ---- tables (constant over k)
  if (kFFT) {
    if (postFull) {
      for (int e = tid; e < L; e += NT) {
        const double2 w = tw[((uint64_t)e * (uint64_t)r2) << a.logR1];  // w_M^{n r2} = w_b^{n r2 R1}
        postLo[e] = mk((Real)w.x, (Real)w.y);
      }
    } else {
      for (int e = tid; e < 128 + 64; e += NT) {
        const uint64_t n = e < 128 ? (uint64_t)e : (uint64_t)(e - 128) << 7;
        if (n < (uint64_t)L) {
          const double2 w = tw[(n * (uint64_t)r2) << a.logR1];
          postLo[e] = mk((Real)w.x, (Real)w.y);
        }
      }
    }
    if (R1 > 1) {
      for (int e = tid; e < cl_pre_hi(a.log2b); e += NT) {
        const uint64_t x = (uint64_t)e << 9;
        const double2 w = x < ((uint64_t)1 << a.log2b) ? tw[x] : make_double2(1.0, 0.0);
        preHi[e] = mk((Real)w.x, (Real)w.y);
      }
      for (int e = tid; e < 512; e += NT) {
        const double2 w = tw[e];
        preLo[e] = mk((Real)w.x, (Real)w.y);
      }
    }
    // pass twiddles w_{8 half}^kk at half = 8^p (FP64: 3 passes after the
    // first) or 16 * 8^(p-1) (FP32), and w_16^k for the cluster combine
    if (!kF32) {
      // [0,8) w_64, [8,72) w_512, [72,584) w_L, [584,592) w_16
      for (int e = tid; e < 8 + 64 + 512 + 8; e += NT) {
        const int lg = e < 8 ? 6 : (e < 72 ? 9 : (e < 584 ? LOGL : 4));
        const int kk = e < 8 ? e : (e < 72 ? e - 8 : (e < 584 ? e - 72 : e - 584));
        const double2 w = tw[(uint32_t)kk << (a.log2b - lg)];
        ptw[e] = mk((Real)w.x, (Real)w.y);
      }
    } else {
      for (int e = tid; e < 16 + 128 + 1024 + 8; e += NT) {
        int lg, kk;
        if (e < 16) { lg = 7; kk = e; }
        else if (e < 144) { lg = 10; kk = e - 16; }
        else if (e < 1168) { lg = 13; kk = e - 144; }
        else { lg = 4; kk = e - 1168; }
        const double2 w = tw[(uint32_t)kk << (a.log2b - lg)];
        ptw[e] = mk((Real)w.x, (Real)w.y);
      }
    }
    for (int e = tid; e < 16; e += NT) {
      const double2 w = e < R1 ? tw[(uint32_t)e << logM] : make_double2(1.0, 0.0);  // w_R1^e
      wRx[e] = (Real)w.x;
      wRy[e] = (Real)w.y;
    }
  }
  auto post = [&](int n) -> C { return postFull ? postLo[n] : cmul(postHi[n >> 7], postLo[n & 127]); };
  // B fragments of H16 for the FP32 FWHT
  uint32_t hb[2][2] = {{0u, 0u}, {0u, 0u}};
  if (!kFFT && kF32) {
    const int gq = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int hf = 0; hf < 2; ++hf) {
      const int c = gq + 8 * hf;
      auto hv = [](int e, int cc) { return (__popc(e & cc) & 1) ? -1.f : 1.f; };
      hb[hf][0] = bf16x2(hv(2 * tq, c), hv(2 * tq + 1, c));
      hb[hf][1] = bf16x2(hv(2 * tq + 8, c), hv(2 * tq + 9, c));
    }
  }

  // the local buffer is cleared once: the scatter writes into it, and the
  // last radix pass of every inner index leaves it zero again
  if (kFFT) {
    for (int e = tid; e < PL; e += NT) buf0[e] = mk((Real)0, (Real)0);
  } else {
    for (int e = tid; e < 2 * PL; e += NT) xs0[e] = (Real)0;
  }
  C* const buf = buf0;
  Real* const xs = xs0;
  Real* const ys = xs0 + PL;
  // exchange slots of this CTA's group in global memory (L2-resident):
  // [parity][R2][L] elements, parity = step & 3
  C* const xgr = reinterpret_cast<C*>(a.xch) + (size_t)blockIdx.y * 4 * (size_t)R2 * L;

  // ---- group barrier of the R2 CTAs of one slab.  The grid is a
  // cooperative launch, so every CTA is resident and every group member
  // arrives.  Each group has one arrival counter per exchange slot (step
  // mod 4); a CTA adds 1 to the counter of step s after its exchange
  // writes, and the wait for step s needs R2 (s / 4 + 1) arrivals there.
  // Counting per slot keeps the wait exact although CTAs drift apart by a
  // step: an arrival at step s + 4 follows its CTA's wait for step s + 2,
  // hence every CTA's arrival at step s.  A wait that runs out of spins
  // sets the host-mapped flag, and this CTA's warps skip their later waits
  // (it still arrives) and it writes NaN partials, so the launch ends in
  // bounded time and the failure is visible.
  unsigned* const gcnt = a.gsync + (size_t)blockIdx.y * 128;  // 4 counters, 128 bytes apart
  __shared__ int s_abort;
  if (tid == 0) s_abort = 0;
  // (called after a barrier that follows this CTA's exchange writes; the
  // release orders them, through that barrier, before the count)
  auto group_arrive = [&](unsigned st) {
    if (tid == 0) red_release_gpu_add(gcnt + (st & 3u) * 32u, 1u);
  };
  // Each warp waits for itself (lane 0 polls with acquire, then the warp
  // synchronises): the combine reads only the other CTAs' global writes and
  // registers, so no CTA-wide barrier is needed, and the warps' round trips
  // to L2 overlap instead of all 16 warps waiting for one thread.
  auto group_wait = [&](unsigned st) {
    if (lane == 0 && !*(volatile int*)&s_abort) {
      const unsigned target = (unsigned)R2 * ((st >> 2) + 1u) + a.wait_extra;
      const unsigned* c = gcnt + (st & 3u) * 32u;
      unsigned spins = 0;
      while (ld_acquire_gpu(c) < target) {
        if (++spins > a.spin_limit) {
          s_abort = 1;
          *a.timeout = 1;
          __threadfence_system();
          break;
        }
        __nanosleep(64);
      }
    }
    __syncwarp();  // after lane 0's acquire: the other CTAs' exchange writes are visible to the warp
  };

  unsigned step = 0;  // inner indices processed by this CTA (selects the exchange slots)
  // ---- persistent loop over work items (r1, t, k-group); every CTA of a
  // group has the same blockIdx.y, hence the same items and barriers
  const int items = (R1 * a.d) * a.G;
  for (int item = blockIdx.y; item < items; item += gridDim.y) {
  const int r1 = item & (R1 - 1);
  const int t = (item >> a.logR1) % a.d;
  const int g = (item >> a.logR1) / a.d;
  __syncthreads();  // the previous item is done with the shared codes and staged rows
  // codes of this CTA's segment, premixed with the DIF weight index for r1
  {
    const CodeT* gA = reinterpret_cast<const CodeT*>(a.codeA) + ((size_t)t * R2 + r2) * a.SA;
    const CodeT* gB = reinterpret_cast<const CodeT*>(a.codeB) + ((size_t)t * R2 + r2) * a.SB;
    for (int64_t e = tid; e < a.SA + a.SB; e += NT) {
      const uint32_t h = e < a.SA ? (uint32_t)gA[e] : (uint32_t)gB[e - a.SA];
      const uint32_t m = h & (L - 1), q1 = h >> LOGL;
      const uint32_t w = kFFT ? ((q1 * (uint32_t)r1) & (uint32_t)(R1 - 1)) : (__popc(q1 & (uint32_t)r1) & 1u);
      (e < a.SA ? cA[e] : cB[e - a.SA]) = (CodeT)(m | (w << LOGL));
    }
  }
  // this thread's contiguous slot range in its segment (compact plan)
  const uint32_t* cutA = a.countA + ((size_t)t * R2 + r2) * (kCT + 1);
  const uint32_t* cutB = a.countB + ((size_t)t * R2 + r2) * (kCT + 1);
  const int begA = (int)cutA[tid * VPT], endA = (int)cutA[(tid + 1) * VPT];
  const int begB = (int)cutB[tid * VPT], endB = (int)cutB[(tid + 1) * VPT];

  // ---- accumulators for this CTA's outputs
  // group gi = tid + NT u (u < OUT / 8) covers sub-spectrum position
  // n = r2 * (L / R2) + (gi >> (logR2 - 3)) and 8 of its R2 outputs
  const int64_t bsz = (int64_t)1 << a.log2b;
  auto out_f = [&](int gi, int jj) -> int64_t {
    const int nl = gi >> (a.logR2 - 3);
    const int half = gi & ((R2 >> 3) - 1);
    const int n = r2 * (L >> a.logR2) + nl;
    if (kFFT) {
      const int j = R2 == 16 ? 2 * jj + half : jj;
      return ((int64_t)n + (int64_t)L * j) * R1 + r1;
    } else {
      const int j = R2 == 16 ? half * 8 + jj : jj;
      return (int64_t)r1 * (bsz >> a.logR1) + (int64_t)n * R2 + j;
    }
  };
  double2* partC = reinterpret_cast<double2*>(a.partial) + ((size_t)g * a.d + t) * (size_t)bsz;
  double* partR = reinterpret_cast<double*>(a.partial) + ((size_t)g * a.d + t) * (size_t)bsz;
  constexpr int QC = kFFT ? 2 : 1;  // components per accumulator
  double qd[OUT][QC];  // FP64 accumulators (FP64 path)
  float qh[OUT][QC], ql[OUT][QC];  // two-sum pairs (FP32 path)
#pragma unroll
  for (int o = 0; o < OUT; ++o) {
    const int gi = tid + NT * (o >> 3);
    const int64_t f = out_f(gi, o & 7);
    double vx = 0.0, vy = 0.0;
    if (a.accumulate) {
      if (kFFT) { const double2 v = partC[f]; vx = v.x; vy = v.y; }
      else vx = partR[f];
    }
    if (kF32) {
      qh[o][0] = (float)vx; ql[o][0] = (float)(vx - (double)qh[o][0]);
      if (kFFT) { qh[o][QC - 1] = (float)vy; ql[o][QC - 1] = (float)(vy - (double)qh[o][QC - 1]); }
    } else {
      qd[o][0] = vx;
      if (kFFT) qd[o][QC - 1] = vy;
    }
  }

  const int64_t per = (a.kc + a.G - 1) / a.G;
  const int64_t kb = (int64_t)g * per;
  const int64_t ke = kb + per < a.kc ? kb + per : a.kc;
  // the next inner index with a nonzero row pair (all-zero rows are skipped
  // identically by every CTA of the group)
  auto next_k = [&](int64_t k) -> int64_t {
    if (kFFT)
      while (k < ke && __ldg(a.scale_exp + a.k0 + k) == kCSkip) ++k;
    return k;
  };
  // stage this CTA's segments of row k, coalesced (thread i copies slots i,
  // i + 512, ...); the copies land before the barrier that precedes the
  // scatter, and are issued after the barrier that ends the previous scatter
  const int totA = (int)cutA[kCT], totB = (int)cutB[kCT];
  auto stage = [&](int64_t k) {
    const Real* rA = reinterpret_cast<const Real*>(a.matA) + (((size_t)t * a.kc + k) * R2 + r2) * a.SA;
    const Real* rB = reinterpret_cast<const Real*>(a.matB) + (((size_t)t * a.kc + k) * R2 + r2) * a.SB;
    for (int e = tid; e < totA; e += NT) {
      if (kF32) cp_async4(stA + spad<Real>(e), rA + e); else cp_async8(stA + spad<Real>(e), rA + e);
    }
    for (int e = tid; e < totB; e += NT) {
      if (kF32) cp_async4(stB + spad<Real>(e), rB + e); else cp_async8(stB + spad<Real>(e), rB + e);
    }
  };

  // ---- scatter the staged row k into the (zero) local buffer.  The plan
  // cuts the segment at bucket boundaries, so every bucket has one writer
  // thread; its slots are sorted by bucket.  Per batch of kCBatch slots a
  // thread loads every target first, sums runs of equal buckets in registers
  // and stores once per run.  The scale is a power of two, applied per value.
  // Side A and side B write different words when the DIF weights are real
  // (FFT with R1 <= 2: real / imaginary part; FWHT: x / y), so both sides
  // run at once.  Ends with a barrier: the buffer is complete and the staged
  // row is free.
  auto scatter = [&](int64_t k) {
    Real alpha = (Real)1, beta = (Real)1;
    if (kFFT) {
      const int se = __ldg(a.scale_exp + a.k0 + k);
      alpha = kF32 ? (Real)__int_as_float((127 - se) << 23) : (Real)__longlong_as_double((long long)(1023 - se) << 52);
      beta = kF32 ? (Real)__int_as_float((127 + se) << 23) : (Real)__longlong_as_double((long long)(1023 + se) << 52);
    }
    const bool split = !kFFT || R1 <= 2;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const Real* st = side == 0 ? stA : stB;
      const CodeT* codes = side == 0 ? cA : cB;
      const int beg = side == 0 ? begA : begB, end = side == 0 ? endA : endB;
      const Real sc = side == 0 ? alpha : beta;
      Real* words = kFFT ? reinterpret_cast<Real*>(buf) + side : (side == 0 ? xs : ys);
      constexpr int kWordStride = kFFT ? 2 : 1;  // Real words per element
      for (int s0 = beg; s0 < end; s0 += kCBatch) {
        Real cx[kCBatch], cy[kCBatch];
        int pp[kCBatch];
        uint32_t mm[kCBatch];
#pragma unroll
        for (int u = 0; u < kCBatch; ++u) {
          const int e = s0 + u;
          const bool ok = e < end;
          const Real v = ok ? st[spad<Real>(e)] * sc : (Real)0;
          const uint32_t h = ok ? (uint32_t)codes[e] : 0u;
          const uint32_t m = h & (L - 1), w = h >> LOGL;
          mm[u] = ok ? m : 0xffffffffu;
          pp[u] = phys<ES>(kFFT ? (int)(__brev(m) >> (32 - LOGL)) : (int)m);
          if (!kFFT) {
            cx[u] = w ? -v : v;
            cy[u] = (Real)0;
          } else if (split) {
            cx[u] = (w & 1u) ? -v : v;  // w_2^w = +-1 (w = 0 when R1 = 1)
            cy[u] = (Real)0;
          } else if (a.logR1 == 2) {  // w_4^w = (-i)^w exactly
            cx[u] = (w & 1u) ? (Real)0 : ((w & 2u) ? -v : v);
            cy[u] = (w & 1u) ? ((w & 2u) ? v : -v) : (Real)0;
          } else {
            cx[u] = v * wRx[w];
            cy[u] = v * wRy[w];
          }
          if (kFFT && !split && side == 1) {  // side B adds i c
            const Real tx = cx[u];
            cx[u] = -cy[u];
            cy[u] = tx;
          }
        }
        if (split) {
          Real old[kCBatch];
#pragma unroll
          for (int u = 0; u < kCBatch; ++u) old[u] = mm[u] != 0xffffffffu ? words[pp[u] * kWordStride] : (Real)0;
          Real rx = (Real)0;
#pragma unroll
          for (int u = 0; u < kCBatch; ++u) {
            rx = (u > 0 && mm[u] == mm[u - 1]) ? rx + cx[u] : cx[u];
            const bool last = u == kCBatch - 1 || mm[u + 1] != mm[u];
            if (mm[u] != 0xffffffffu && last) words[pp[u] * kWordStride] = old[u] + rx;
          }
        } else {
          C old[kCBatch];
#pragma unroll
          for (int u = 0; u < kCBatch; ++u) old[u] = mm[u] != 0xffffffffu ? buf[pp[u]] : mk((Real)0, (Real)0);
          Real rx = (Real)0, ry = (Real)0;
#pragma unroll
          for (int u = 0; u < kCBatch; ++u) {
            const bool cont = u > 0 && mm[u] == mm[u - 1];
            rx = cont ? rx + cx[u] : cx[u];
            ry = cont ? ry + cy[u] : cy[u];
            const bool last = u == kCBatch - 1 || mm[u + 1] != mm[u];
            if (mm[u] != 0xffffffffu && last) buf[pp[u]] = mk(old[u].x + rx, old[u].y + ry);
          }
        }
      }
      if (side == 0 && !split) __syncthreads();
    }
    __syncthreads();  // the buffer is complete; the staged row is free
  };

  // ---- local transform of length L in shared memory.  The last pass
  // writes the sub-spectrum to this CTA's exchange slot xo (natural order;
  // FWHT: (x, y) pairs) and zeros to the buffer.
  auto transform = [&](C* __restrict__ xo) {
    if (kFFT && !kF32 && NT != kCT) {
      // L = 2048, 256 threads: 3 radix-8 DIT passes (pass 0 applies the DIF
      // weight w_b^{n1 r1}, r1 > 0) and a radix-4 pass of two butterflies
      // per thread that applies the post-twiddle w_M^{n r2}
#pragma unroll
      for (int ps = 0; ps < 3; ++ps) {
        const int s0 = 3 * ps, half = 1 << s0;
        const int kk2 = tid & (half - 1);
        const int base = ((tid >> s0) << (s0 + 3)) | kk2;
        C x[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) x[e] = buf[phys<ES>(base + e * half)];
        if (ps == 0) {
          if (r1 > 0) {
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const uint32_t m = __brev((uint32_t)(base + e)) >> (32 - LOGL);
              const uint32_t xx = ((m << a.logR2) + (uint32_t)r2) * (uint32_t)r1;  // n1 r1 < b
              x[e] = cmul(x[e], cmul(preHi[xx >> 9], preLo[xx & 511]));
            }
          }
          r8_first(x);
        } else {
          r8(x, ptw[(ps == 1 ? 0 : 8) + kk2]);
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) buf[phys<ES>(base + e * half)] = x[e];
        __syncthreads();
      }
#pragma unroll
      for (int gg = 0; gg < 2; ++gg) {
        const int p = tid + gg * NT;  // butterfly p < 512 at half = 512: points p + 512 e
        C x[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) x[e] = buf[phys<ES>(p + e * 512)];
        r4(x, ptw[72 + p]);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int n = p + e * 512;
          __stcg(xo + n, r2 > 0 ? cmul(x[e], post(n)) : x[e]);
          buf[phys<ES>(n)] = mk((Real)0, (Real)0);
        }
      }
    } else if (kFFT && !kF32) {
      // 4 radix-8 DIT passes; pass 0 (constant twiddles) applies the DIF
      // weight w_b^{n1 r1} (r1 > 0), pass 3 the post-twiddle w_M^{n r2}
#pragma unroll
      for (int ps = 0; ps < 4; ++ps) {
        const int s0 = 3 * ps, half = 1 << s0;
        const int kk2 = tid & (half - 1);
        const int base = ((tid >> s0) << (s0 + 3)) | kk2;
        C x[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) x[e] = buf[phys<ES>(base + e * half)];
        if (ps == 0) {
          if (r1 > 0) {
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const uint32_t m = __brev((uint32_t)(base + e)) >> (32 - LOGL);
              const uint32_t xx = ((m << a.logR2) + (uint32_t)r2) * (uint32_t)r1;  // n1 r1 < b
              x[e] = cmul(x[e], cmul(preHi[xx >> 9], preLo[xx & 511]));
            }
          }
          r8_first(x);
        } else {
          r8(x, ptw[(ps == 1 ? 0 : (ps == 2 ? 8 : 72)) + kk2]);
        }
        if (ps == 3) {
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const int n = base + e * half;
            __stcg(xo + n, r2 > 0 ? cmul(x[e], post(n)) : x[e]);
            buf[phys<ES>(n)] = mk((Real)0, (Real)0);
          }
        } else {
#pragma unroll
          for (int e = 0; e < 8; ++e) buf[phys<ES>(base + e * half)] = x[e];
          __syncthreads();
        }
      }
    } else if (kFFT) {
      // FP32, L = 8192: radix-16 (stages 0-3) + 3 radix-8 passes
      {
        const int base = tid * 16;
        C x[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) x[e] = buf[phys<ES>(base + e)];
        if (r1 > 0) {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const uint32_t m = __brev((uint32_t)(base + e)) >> (32 - LOGL);
            const uint32_t xx = ((m << a.logR2) + (uint32_t)r2) * (uint32_t)r1;
            x[e] = cmul(x[e], cmul(preHi[xx >> 9], preLo[xx & 511]));
          }
        }
        // stages 0 and 1 have the twiddles 1 and -i
#pragma unroll
        for (int e = 0; e < 16; e += 2) add_sub(x[e], x[e + 1]);
#pragma unroll
        for (int e = 0; e < 16; e += 4) {
          add_sub(x[e], x[e + 2]);
          x[e + 3] = mul_mi(x[e + 3]);
          add_sub(x[e + 1], x[e + 3]);
        }
#pragma unroll
        for (int st = 2; st < 4; ++st) {
          const int hh = 1 << st;
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            if (e & hh) continue;
            bf(x[e], x[e + hh], ptw[1168 + (e & (hh - 1)) * (8 >> st)]);
          }
        }
#pragma unroll
        for (int e = 0; e < 16; ++e) buf[phys<ES>(base + e)] = x[e];
      }
      __syncthreads();
#pragma unroll
      for (int ps = 1; ps <= 3; ++ps) {
        const int s0 = ps == 1 ? 4 : (ps == 2 ? 7 : 10), half = 1 << s0;
#pragma unroll
        for (int gg = 0; gg < 2; ++gg) {
          const int gi = tid + gg * NT;
          const int kk2 = gi & (half - 1);
          const int base = ((gi >> s0) << (s0 + 3)) | kk2;
          C x[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) x[e] = buf[phys<ES>(base + e * half)];
          r8(x, ptw[(ps == 1 ? 0 : (ps == 2 ? 16 : 144)) + kk2]);
          if (ps == 3) {
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const int n = base + e * half;
              __stcg(xo + n, r2 > 0 ? cmul(x[e], post(n)) : x[e]);
              buf[phys<ES>(n)] = mk((Real)0, (Real)0);
            }
          } else {
#pragma unroll
            for (int e = 0; e < 8; ++e) buf[phys<ES>(base + e * half)] = x[e];
          }
        }
        if (ps < 3) __syncthreads();
      }
    } else if (!kF32 && NT != kCT) {
      // FP64 WHT of x and y, L = 4096, 256 threads, three radix-16 passes
      // (the stages of a WHT commute): index bits 8-11, bits 0-3, then bits
      // 4-7, whose pass writes the exchange slot as (x, y) pairs
#pragma unroll
      for (int gg = 0; gg < 2; ++gg) {
        Real* arr = gg == 0 ? xs : ys;
        Real v[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) v[e] = arr[phys<ES>(tid + e * 256)];
        whtr<Real, 16>(v);
#pragma unroll
        for (int e = 0; e < 16; ++e) arr[phys<ES>(tid + e * 256)] = v[e];
      }
      __syncthreads();
#pragma unroll
      for (int gg = 0; gg < 2; ++gg) {
        Real* arr = gg == 0 ? xs : ys;
        const int base = tid * 16;
        Real v[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) v[e] = arr[phys<ES>(base + e)];
        whtr<Real, 16>(v);
#pragma unroll
        for (int e = 0; e < 16; ++e) arr[phys<ES>(base + e)] = v[e];
      }
      __syncthreads();
      {
        const int base = ((tid >> 4) << 8) | (tid & 15);
        Real x[16], y[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) { x[e] = xs[phys<ES>(base + e * 16)]; y[e] = ys[phys<ES>(base + e * 16)]; }
        whtr<Real, 16>(x);
        whtr<Real, 16>(y);
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int n = base + e * 16;
          __stcg(xo + n, mk(x[e], y[e]));
          xs[phys<ES>(n)] = (Real)0;
          ys[phys<ES>(n)] = (Real)0;
        }
      }
    } else if (!kF32 || !a.tc) {
      // WHT of x and y (FP64, or FP32 on CUDA cores) in three passes over
      // shared memory (the stages of a WHT commute): index bits 8-12 (radix
      // 32, one array per thread), bits 0-3, then bits 4-7, whose pass
      // writes the exchange slot as (x, y) pairs, contiguous per half-warp
      {
        Real* arr = tid < 256 ? xs : ys;
        const int base = tid & 255;
        Real v[32];
#pragma unroll
        for (int e = 0; e < 32; ++e) v[e] = arr[phys<ES>(base + e * 256)];
        whtr<Real, 32>(v);
#pragma unroll
        for (int e = 0; e < 32; ++e) arr[phys<ES>(base + e * 256)] = v[e];
      }
      __syncthreads();
#pragma unroll
      for (int gg = 0; gg < 2; ++gg) {
        Real* arr = gg == 0 ? xs : ys;
        const int base = tid * 16;
        Real v[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) v[e] = arr[phys<ES>(base + e)];
        whtr<Real, 16>(v);
#pragma unroll
        for (int e = 0; e < 16; ++e) arr[phys<ES>(base + e)] = v[e];
      }
      __syncthreads();
      {
        const int base = ((tid >> 4) << 8) | (tid & 15);
        Real x[16], y[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) { x[e] = xs[phys<ES>(base + e * 16)]; y[e] = ys[phys<ES>(base + e * 16)]; }
        whtr<Real, 16>(x);
        whtr<Real, 16>(y);
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int n = base + e * 16;
          __stcg(xo + n, mk(x[e], y[e]));
          xs[phys<ES>(n)] = (Real)0;
          ys[phys<ES>(n)] = (Real)0;
        }
      }
    } else {
      // FP32 WHT: three Hadamard-16 factors on the tensor cores + radix-2
      float* fx = reinterpret_cast<float*>(xs);
      float* fy = reinterpret_cast<float*>(ys);
      h16<0>(fx, hb, warp, lane);
      h16<0>(fy, hb, warp, lane);
      __syncthreads();
      h16<1>(fx, hb, warp, lane);
      h16<1>(fy, hb, warp, lane);
      __syncthreads();
      h16<2>(fx, hb, warp, lane);
      h16<2>(fy, hb, warp, lane);
      __syncthreads();
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int m = tid + NT * e;
        const float x0 = fx[phys<ES>(m)], x1 = fx[phys<ES>(m + 4096)];
        const float y0 = fy[phys<ES>(m)], y1 = fy[phys<ES>(m + 4096)];
        __stcg(xo + m, mk((Real)(x0 + x1), (Real)(y0 + y1)));
        __stcg(xo + m + 4096, mk((Real)(x0 - x1), (Real)(y0 - y1)));
        fx[phys<ES>(m)] = 0.f; fx[phys<ES>(m + 4096)] = 0.f;
        fy[phys<ES>(m)] = 0.f; fy[phys<ES>(m + 4096)] = 0.f;
      }
    }
  };

  // ---- radix-R2 combine of the group's sub-spectra, read back from the
  // exchange slots xst of this step; accumulate.  With R2 = 16 the two
  // threads of a lane pair own the even / odd outputs of one position: each
  // reads half of the 16 sub-spectra and they swap halves by shuffle.
  auto combine = [&](const C* __restrict__ xst) {
#pragma unroll
    for (int u = 0; u < OUT / 8; ++u) {
      const int gi = tid + NT * u;
      const int nl = gi >> (a.logR2 - 3);
      const int half = gi & ((R2 >> 3) - 1);
      const int n = r2 * (L >> a.logR2) + nl;
      const int rb = (R2 == 16 && half) ? 8 : 0;
      C z[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) z[r] = __ldcg(xst + (size_t)(rb + r) * L + n);
      if (kFFT) {
        if (R2 == 16) {
#pragma unroll
          for (int r = 0; r < 8; ++r) {
            const C o = mk(__shfl_xor_sync(0xffffffffu, z[r].x, 1), __shfl_xor_sync(0xffffffffu, z[r].y, 1));
            // even outputs: z_r + z_{r+8}; odd outputs: w_16^r (z_r - z_{r+8})
            if (half == 0) z[r] = mk(z[r].x + o.x, z[r].y + o.y);
            else z[r] = cmul(mk(o.x - z[r].x, o.y - z[r].y), ptw[(kF32 ? 1168 : 584) + r]);
          }
        }
        dft8(z);
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const int o = u * 8 + jj;
          const Real zr = z[jj].x * z[jj].x - z[jj].y * z[jj].y;
          const Real zi = (z[jj].x + z[jj].x) * z[jj].y;
          if (kF32) {
            tsum(qh[o][0], ql[o][0], (float)zr);
            tsum(qh[o][QC - 1], ql[o][QC - 1], (float)zi);
          } else {
            qd[o][0] += (double)zr;
            qd[o][QC - 1] += (double)zi;
          }
        }
      } else {
        Real zx[8], zy[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) { zx[r] = z[r].x; zy[r] = z[r].y; }
        if (R2 == 16) {
#pragma unroll
          for (int r = 0; r < 8; ++r) {
            const Real ox = __shfl_xor_sync(0xffffffffu, zx[r], 1), oy = __shfl_xor_sync(0xffffffffu, zy[r], 1);
            zx[r] = half == 0 ? zx[r] + ox : ox - zx[r];
            zy[r] = half == 0 ? zy[r] + oy : oy - zy[r];
          }
        }
        whtr<Real, 8>(zx);
        whtr<Real, 8>(zy);
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const int o = u * 8 + jj;
          if (kF32) tsum(qh[o][0], ql[o][0], (float)(zx[jj] * zy[jj]));
          else qd[o][0] = fma((double)zx[jj], (double)zy[jj], qd[o][0]);
        }
      }
    }
  };

  // ---- software pipeline over the inner indices.  On entry to an
  // iteration row kk is scattered in the buffer and row kn is being staged.
  // Iteration i transforms row i and writes its sub-spectrum, scatters row
  // i + 1, arrives for step i, and only then waits for step i - 1 and
  // combines it: an iteration separates each arrival from the wait that
  // needs it.
  // The exchange slots rotate over four parities (step mod 4): a CTA writes
  // the slot of step i after its wait for step i - 2, which follows every
  // CTA's arrival at step i - 2, which follows that CTA's combine of step
  // i - 4, the last reader of the slot.
  int64_t kk = next_k(kb);
  int64_t kn = ke;
  if (kk < ke) {
    stage(kk);
    cp_async_wait_all();
    __syncthreads();
    scatter(kk);
    kn = next_k(kk + 1);
    if (kn < ke) stage(kn);
  }
#ifdef CMM_PHASE_CLOCKS
  long long t_ph = 0;
#endif
  const C* pend = nullptr;  // exchange slots of the step whose combine is pending
  while (kk < ke) {
    CL_MARK(-1);
    // the row after next, looked up now: the load's latency hides behind
    // the transform
    const int64_t k2 = kn < ke ? next_k(kn + 1) : ke;
    C* const xst = xgr + (size_t)(step & 3) * R2 * L;
    transform(xst + (size_t)r2 * L);
    CL_MARK(0);
    if (kn < ke) {
      cp_async_wait_all();  // this thread's copies of row kn; the barrier publishes all
      __syncthreads();      // (and the transform's exchange writes are all issued)
      CL_MARK(1);
      scatter(kn);
      CL_MARK(2);
    } else {
      __syncthreads();
    }
    // arrive after the scatter, and wait for the previous index: the
    // readers of this step wait for it only in the next iteration.  The
    // next row is staged after the combine, so that its copies sit in front
    // of neither thread 0's barrier traffic nor the combine's loads.
    group_arrive(step);
    if (pend) group_wait(step - 1u);
    CL_MARK(3);
    if (pend) combine(pend);
    CL_MARK(4);
    if (k2 < ke) stage(k2);  // overlaps the next transform
#ifdef CMM_PHASE_CLOCKS
    if (tid == 0) atomicAdd(&g_cl_phase[kClPhases], 1ull);
#endif
    pend = xst;
    ++step;
    kk = kn;
    kn = k2;
  }
  if (pend) {  // the item's last step
    group_wait(step - 1u);
    combine(pend);
  }

  __syncthreads();  // every warp's waits of this item are done
  const bool bad = s_abort != 0;
#pragma unroll
  for (int o = 0; o < OUT; ++o) {
    const int gi = tid + NT * (o >> 3);
    const int64_t f = out_f(gi, o & 7);
    double vx = kF32 ? (double)qh[o][0] + (double)ql[o][0] : qd[o][0];
    double vy = kF32 ? (double)qh[o][QC - 1] + (double)ql[o][QC - 1] : qd[o][QC - 1];
    if (bad) vx = vy = __longlong_as_double(0x7ff8000000000000ll);
    if (kFFT) partC[f] = make_double2(vx, vy);
    else partR[f] = vx;
  }
  }  // item loop
}

// ------------------------------------------------------------------ host
// Sums of the per-phase cycles over all CTAs and inner indices since the
// last call, and the number of (CTA, inner index) steps timed; false when
// the library was built without CMM_PHASE_CLOCKS.
bool cluster_phase_cycles(double* cycles, double* steps) {
#ifdef CMM_PHASE_CLOCKS
  unsigned long long h[kClPhases + 1];
  CMM_CUDA(cudaDeviceSynchronize());
  CMM_CUDA(cudaMemcpyFromSymbol(h, g_cl_phase, sizeof(h)));
  const unsigned long long zero[kClPhases + 1] = {};
  CMM_CUDA(cudaMemcpyToSymbol(g_cl_phase, zero, sizeof(zero)));
  for (int i = 0; i < kClPhases; ++i) cycles[i] = (double)h[i];
  *steps = (double)h[kClPhases];
  return true;
#else
  for (int i = 0; i < kClPhases; ++i) cycles[i] = 0.0;
  *steps = 0.0;
  return false;
#endif
}

static int cl_logL(int variant, bool f32, int nt) {
  return ((variant == kVariantFFT && !f32) ? 12 : 13) - (nt == kCT ? 0 : 1);
}

bool sketch_cluster_applicable(int variant, bool f32, int b) {
  const int logL = cl_logL(variant, f32, kCT);
  int log2b = 0;
  while ((1 << log2b) < b) ++log2b;
  return log2b - logL >= 3 && log2b <= 19;  // R >= 8; DIF twiddle table covers b <= 2^19
}

constexpr size_t kClSmemMax = 227 * 1024 - 64;  // less the kernel's static shared bytes

template <int V, typename Real, typename CodeT, int NT>
static void cl_kernel_attrs(size_t smem) {
  CMM_CUDA(cudaFuncSetAttribute(k_sketch_cluster<V, Real, CodeT, NT>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
}

// shared bytes of one CTA
// (FP64 FFT: the full post-twiddle table when it fits, else the factored one)
static size_t cl_smem(int variant, bool f32, bool u16, int logL, int R1, int log2b, int64_t SA, int64_t SB,
                      bool* post_full = nullptr) {
  const bool fft = variant == kVariantFFT;
  if (fft && !f32 && logL == cl_logL(variant, f32, kCT)) {  // 512-thread form: one CTA per SM
    const size_t full = cl_layout(fft, f32, u16, logL, R1, log2b, SA, SB, true).total;
    if (full <= kClSmemMax) {
      if (post_full) *post_full = true;
      return full;
    }
  }
  if (post_full) *post_full = false;
  return cl_layout(fft, f32, u16, logL, R1, log2b, SA, SB, false).total;
}

// cooperative launch: the group barriers need every CTA resident
template <int V, typename Real, typename CodeT, int NT>
static void cl_launch(const ClArgs& a, dim3 grid, size_t smem, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(NT, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CMM_CUDA(cudaLaunchKernelEx(&cfg, k_sketch_cluster<V, Real, CodeT, NT>, a));
}

// CTAs resident on the whole device at this shared-memory size
template <int V, typename Real, typename CodeT, int NT>
static int cl_resident_t(size_t smem) {
  cl_kernel_attrs<V, Real, CodeT, NT>(smem);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sketch_cluster<V, Real, CodeT, NT>, NT, smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return per_sm * num_sms();
}
static int cl_resident_query(int variant, bool f32, int nt, size_t smem) {
  if (variant == kVariantFFT) {
    if (f32) return cl_resident_t<0, float, uint16_t, kCT>(smem);
    return nt == kCT ? cl_resident_t<0, double, uint16_t, kCT>(smem) : cl_resident_t<0, double, uint16_t, kCT / 2>(smem);
  }
  if (f32) return cl_resident_t<1, float, uint16_t, kCT>(smem);
  return nt == kCT ? cl_resident_t<1, double, uint16_t, kCT>(smem) : cl_resident_t<1, double, uint16_t, kCT / 2>(smem);
}
// the same, cached per (device, variant, precision, threads, shared bytes):
// the occupancy query costs milliseconds of host time
static int cl_resident(int variant, bool f32, int nt, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, int, size_t>, int> cache;
  int dev = 0;
  CMM_CUDA(cudaGetDevice(&dev));
  const auto key = std::make_tuple(dev, variant, (int)f32, nt, smem);
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  const int n = cl_resident_query(variant, f32, nt, smem);
  std::lock_guard<std::mutex> g(mu);
  cache[key] = n;
  return n;
}

// host-mapped flag set by a group wait that ran out of spins
static int* group_timeout_flag(int** dev) {
  static int* host = nullptr;
  static int* mapped = nullptr;
  static std::mutex mu;
  std::lock_guard<std::mutex> g(mu);
  if (!host) {
    CMM_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&host), sizeof(int), cudaHostAllocMapped));
    *host = 0;
    CMM_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&mapped), host, 0));
  }
  if (dev) *dev = mapped;
  return host;
}

bool sketch_group_timed_out() {
  volatile int* h = group_timeout_flag(nullptr);
  const bool t = *h != 0;
  *h = 0;
  return t;
}

// FP32 FWHT stages: CUDA-core passes (default: measured on B200 at
// n = 16384, b = 2^18, d = 9, 237 against 412 ms of sketch kernel per
// product for the tensor-core Hadamard-16 stages with the BF16 hi/mid/lo
// split, whose three products per tile cost more than the adds they
// replace) or the tensor-core stages; CMM_MIXED_WHT=tc|cuda overrides
static bool mixed_wht_tensor_cores() {
  static const bool tc = [] {
    const char* e = getenv("CMM_MIXED_WHT");
    return e && !strcmp(e, "tc");
  }();
  return tc;
}

// threads per CTA of the FP64 group kernels: CMM_GROUP_THREADS=512|256
// overrides the default
static int group_threads(bool f32) {
  if (f32) return kCT;
  static const int nt = [] {
    const char* e = getenv("CMM_GROUP_THREADS");
    if (e && atoi(e) == kCT / 2) return kCT / 2;
    if (e && atoi(e) == kCT) return kCT;
    return kCT;
  }();
  return nt;
}

// Chooses R2 in {16, 8} and the k-group count G from the number of groups
// NG = resident CTAs / R2: the grid holds NG persistent groups that share
// the R1 * d * G work items round-robin; the estimate ceil(items/NG)/G is
// minimised (ties to R2 = 16: less scatter redundancy, fewer items).
// 256-thread CTAs are used only when two of them fit on an SM.
ClusterPlan plan_cluster(int variant, bool f32, int64_t n_inner, int d, int b, int64_t n_a, int64_t n_b) {
  ClusterPlan C;
  C.nt = group_threads(f32);
  C.log2b = 0;
  while ((1 << C.log2b) < b) ++C.log2b;
  for (int attempt = 0; attempt < 2; ++attempt) {
    C.logL = cl_logL(variant, f32, C.nt);
    const int logR = C.log2b - C.logL;
    double best = 1e300;
    for (int logR2 : {4, 3}) {
      if (logR2 > logR) continue;
      const int R2 = 1 << logR2, R1 = 1 << (logR - logR2);
      // a CTA's segment: the indices of one residue class, n / R2 on
      // average; the estimate allows four standard deviations (the launch
      // checks the actual sizes)
      auto seg = [&](int64_t n) {
        const double m = (double)n / R2;
        return (int64_t)(m + 4.0 * std::sqrt(m) + 64.0);
      };
      const size_t smem = cl_smem(variant, f32, true, C.logL, R1, C.log2b, seg(n_a), seg(n_b));
      if (smem > kClSmemMax) continue;
      const int ctas = cl_resident(variant, f32, C.nt, smem);
      if (C.nt != kCT && ctas < 2 * num_sms()) continue;
      const int mx = ctas / R2;
      if (mx <= 0) continue;
      const int64_t base = (int64_t)R1 * d;
      for (int64_t G = 1; G <= 64; ++G) {
        if (G > 1 && G > n_inner) break;
        if (base * G > 65535) break;
        const int64_t items = base * G;
        const int64_t nc = items < mx ? items : mx;
        // per-group load in units of one (r1, t) over all k; scatter cost ~R1
        const double load = (double)((items + nc - 1) / nc) / (double)G * (1.0 + 0.05 * R1);
        if (load < best - 1e-9) {
          best = load;
          C.logR2 = logR2;
          C.logR1 = logR - logR2;
          C.G = (int)G;
          C.max_clusters = (int)nc;
        }
      }
    }
    if (best < 1e299) break;
    if (C.nt == kCT) throw unsupported("no group configuration fits this device");
    C.nt = kCT;  // two 256-thread CTAs do not fit an SM: one of 512
  }
  if (getenv("CMM_DEBUG"))
    fprintf(stderr, "[cmm] group plan: b=%d L=%d R1=%d R2=%d G=%d groups=%d threads=%d\n", b, 1 << C.logL,
            1 << C.logR1, 1 << C.logR2, C.G, C.max_clusters, C.nt);
  return C;
}

bool cluster_smem_fits(int variant, bool f32, const ClusterPlan& C, const SlabPlan& P) {
  return cl_smem(variant, f32, P.u16, C.logL, 1 << C.logR1, C.log2b, P.EA, P.EB) <= kClSmemMax;
}

void launch_sketch_cluster(int variant, bool f32, const ClusterPlan& C, const SlabPlan& P,
                           const void* dMatA, const void* dMatB, int64_t kc, const int* dScaleExp,
                           int64_t k0, const double2* dTw, void* dPartial, int d, int accumulate,
                           cudaStream_t s) {
  ClArgs a;
  a.matA = dMatA;
  a.matB = dMatB;
  a.codeA = P.codeA.ptr;
  a.codeB = P.codeB.ptr;
  a.countA = P.countA.as<uint32_t>();
  a.countB = P.countB.as<uint32_t>();
  a.scale_exp = dScaleExp;
  a.tw = dTw;
  a.partial = dPartial;
  a.SA = P.EA;  // compact segments
  a.SB = P.EB;
  a.kc = kc;
  a.k0 = k0;
  a.d = d;
  a.log2b = C.log2b;
  a.logR1 = C.logR1;
  a.logR2 = C.logR2;
  a.G = C.G;
  a.accumulate = accumulate;
  const int R2 = 1 << C.logR2, R1 = 1 << C.logR1;
  bool post_full = false;
  const size_t smem = cl_smem(variant, f32, P.u16, C.logL, R1, C.log2b, a.SA, a.SB, &post_full);
  a.post_full = post_full ? 1 : 0;
  if (smem > kClSmemMax) throw unsupported("cluster sketch: residue segments too large for shared memory");
  if (sketch_group_timed_out())
    throw std::runtime_error("cluster sketch: a group barrier wait ran out in an earlier launch");
  // exchange area: four parities of R2 sub-spectra of L elements per group;
  // arrival counters: four per group, one 128-byte line each
  const size_t elem = f32 ? 8 : 16;
  // every CTA must be resident (cooperative launch): the actual segment
  // sizes can need more shared memory than the plan's estimate
  const int groups = std::min(C.max_clusters, cl_resident(variant, f32, C.nt, smem) / R2);
  if (groups < 1) throw unsupported("cluster sketch: no group of CTAs fits the device");
  DevBuf xch((size_t)groups * 4 * (size_t)R2 * ((size_t)1 << C.logL) * elem, s);
  DevBuf gsync((size_t)groups * 512, s);
  CMM_CUDA(cudaMemsetAsync(gsync.ptr, 0, gsync.bytes, s));
  a.xch = xch.ptr;
  a.gsync = gsync.as<unsigned>();
  group_timeout_flag(&a.timeout);
  a.spin_limit = 1u << 24;  // over a second of 64 ns sleeps; a step takes microseconds
  a.wait_extra = 0;
  a.tc = mixed_wht_tensor_cores() ? 1 : 0;
  if (const char* e = getenv("CMM_TEST_GROUP_WAIT_EXTRA")) {  // test hook: waits that cannot complete
    a.wait_extra = (unsigned)atoi(e);
    if (a.wait_extra) a.spin_limit = 2000;
  }
  if (getenv("CMM_DEBUG"))
    fprintf(stderr, "[cmm] group launch: smem=%zu SA=%lld SB=%lld groups=%d threads=%d exchange=%zu bytes\n",
            smem, (long long)a.SA, (long long)a.SB, groups, C.nt, xch.bytes);
  const dim3 grid((unsigned)R2, (unsigned)groups, 1);
  ProfScope prof("sketch", s);
  count_launch();
#define CMM_CL(V, T, CT, NT)                   \
  do {                                         \
    cl_kernel_attrs<V, T, CT, NT>(smem);       \
    cl_launch<V, T, CT, NT>(a, grid, smem, s); \
  } while (0)
  const bool half = C.nt != kCT;
  if (half && f32) throw std::logic_error("256-thread group kernels are FP64 only");
  if (variant == kVariantFFT) {
    if (f32) { if (P.u16) CMM_CL(0, float, uint16_t, kCT); else CMM_CL(0, float, uint32_t, kCT); }
    else if (half) { if (P.u16) CMM_CL(0, double, uint16_t, kCT / 2); else CMM_CL(0, double, uint32_t, kCT / 2); }
    else { if (P.u16) CMM_CL(0, double, uint16_t, kCT); else CMM_CL(0, double, uint32_t, kCT); }
  } else {
    if (f32) { if (P.u16) CMM_CL(1, float, uint16_t, kCT); else CMM_CL(1, float, uint32_t, kCT); }
    else if (half) { if (P.u16) CMM_CL(1, double, uint16_t, kCT / 2); else CMM_CL(1, double, uint32_t, kCT / 2); }
    else { if (P.u16) CMM_CL(1, double, uint16_t, kCT); else CMM_CL(1, double, uint32_t, kCT); }
  }
#undef CMM_CL
  CMM_CUDA(cudaGetLastError());
}

}  // namespace cmm
