// Batched natural-order Walsh-Hadamard transform of FP32 rows, with the two
// Hadamard-16 stages on the 5th-generation tensor cores (tcgen05.mma: BF16
// operands from shared memory, FP32 accumulators in tensor memory), beside
// the same transform with every stage on CUDA cores.
//
// y[r] = H_L x[r] for each row r, L = 2^LOGL (11 <= LOGL <= 13), H_L the
// unnormalised Sylvester matrix H[i][j] = (-1)^popc(i & j): the forward
// transform of the reference's fwht_transformer (transform.hpp:94-144, FXT
// walsh_wak in natural order; golden values in tests.cpp:621-671).
//
// H_L = H_{L/256} (x) H_16 (x) H_16 acting on the index bits [8, LOGL),
// [4, 8) and [0, 4).  The three factors commute:
//   stage 1 (bits 0-3): X seen as an (L/16) x 16 matrix whose row m holds
//     elements 16 m .. 16 m + 15; X <- X H16.
//   stage 2 (bits 4-7): row m = 16 blk + j holds elements 256 blk + 16 i + j
//     (i = 0..15); the same product on that view.
//   stage 3 (bits 8+): L/256-point transforms at stride 256, CUDA cores.
//
// Tensor-core form of stages 1-2.  Every FP32 value is split into BF16
// hi + mid + lo (each part the round-to-nearest BF16 of what the earlier
// parts leave; the sum equals x to about 2^-27 |x|).  Per 128-row tile three
// MMAs (M = 128, N = 16, K = 16) accumulate A_hi H + A_mid H + A_lo H into one
// FP32 accumulator of 16 TMEM columns; H is exact in BF16, so the products
// are exact and only the FP32 accumulation rounds, as in the CUDA-core
// butterflies.  The A tiles sit in shared memory in the no-swizzle K-major
// core-matrix layout: element (m, k) at byte (m / 8) * 256 + (k / 8) * 128 +
// (m % 8) * 16 + (k % 8) * 2 (8 x 16-byte core matrices; 128 B between the
// two K halves, 256 B between 8-row groups).  One elected thread issues the
// MMAs and commits them to an mbarrier; each warp then reads its 32 TMEM
// lanes (tcgen05.ld 32x32b.x16) and writes the results back in place.
//
// Shared layout of a row: X[phys(e)], phys(e) = e + 4 (e / 32), which keeps
// the 16-byte accesses of stage 1 and the strided accesses of stages 2-3
// free of bank conflicts.
//
// Waits: the mbarrier wait of each tensor-core stage is bounded; when it
// runs out the CTA records a timeout in a host-mapped flag, waits (bounded)
// once more for the MMAs it issued, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include <mutex>

#include "cmm_fft_device.cuh"
#include "cmm_internal.h"

namespace cmm {
namespace {

constexpr int kWT = 128;                 // threads per CTA: one per TMEM lane of a tile
constexpr uint32_t kWaitSpins = 1u << 22;  // polls before a stage gives up

__device__ __forceinline__ int phys(int e) { return e + ((e >> 5) << 2); }
__host__ __device__ constexpr int phys_len(int L) { return L + L / 8; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// byte offset of element (m, k) in the K-major core-matrix layout (m < L/16, k < 16)
__device__ __forceinline__ int a_off(int m, int k) {
  return ((m >> 3) << 8) + ((k >> 3) << 7) + ((m & 7) << 4) + ((k & 7) << 1);
}
// shared-memory matrix descriptor (sm_100 form): start address >> 4, leading
// byte offset 128 (between the K halves), stride byte offset 256 (between
// 8-row groups), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
         (1ull << 46);
}
// instruction descriptor, kind::f16: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 and 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// non-blocking polls with short sleeps: at most kWaitSpins polls (about half a
// second), whatever the MMAs do
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < kWaitSpins; ++it) {
    if (mbar_test_wait(bar, parity)) return true;
    __nanosleep(32);
  }
  return false;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int e = 0; e < 16; ++e) v[e] = __uint_as_float(r[e]);
}

// x -> hi + mid + lo in BF16 (x - hi and the next residual are exact in FP32)
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& mid, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(hi);
  mid = __float2bfloat16_rn(r1);
  lo = __float2bfloat16_rn(r1 - __bfloat162float(mid));
}

// element e of the 16-wide row m in stage s (1: 16 m + k; 2: 256 blk + 16 k + j)
template <int S>
__device__ __forceinline__ int stage_elem(int m, int k) {
  return S == 1 ? 16 * m + k : ((m >> 4) << 8) + 16 * k + (m & 15);
}

// CUDA-core Hadamard-16 stage S on X (each thread transforms whole 16-rows)
template <int LOGL, int S>
__device__ __forceinline__ void cc_stage16(float* X, int tid) {
  constexpr int MR = (1 << LOGL) / 16;
  for (int m = tid; m < MR; m += kWT) {
    float v[16];
    if (S == 1) {
      const float4* p = reinterpret_cast<const float4*>(X + phys(16 * m));
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float4 f = p[q];
        v[4 * q] = f.x, v[4 * q + 1] = f.y, v[4 * q + 2] = f.z, v[4 * q + 3] = f.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) v[k] = X[phys(stage_elem<2>(m, k))];
    }
    dev::whtr<float, 16>(v);
    if (S == 1) {
      float4* p = reinterpret_cast<float4*>(X + phys(16 * m));
#pragma unroll
      for (int q = 0; q < 4; ++q) p[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) X[phys(stage_elem<2>(m, k))] = v[k];
    }
  }
}

// stage 3: L/256-point transforms over stride 256 (columns c < 256)
template <int LOGL>
__device__ __forceinline__ void cc_stage_hi(float* X, int tid) {
  constexpr int F = (1 << LOGL) / 256;
  for (int c = tid; c < 256; c += kWT) {
    float v[F];
#pragma unroll
    for (int f = 0; f < F; ++f) v[f] = X[phys(c + 256 * f)];
    dev::whtr<float, F>(v);
#pragma unroll
    for (int f = 0; f < F; ++f) X[phys(c + 256 * f)] = v[f];
  }
}

// Tensor-core Hadamard-16 stage S.  Returns false (uniformly over the CTA)
// when the MMA completion wait ran out; *parity is the phase awaited next.
template <int LOGL, int S>
__device__ __forceinline__ bool tc_stage16(float* X, unsigned char* As, const unsigned char* Bs, uint32_t tbase,
                                           uint64_t* bar, uint32_t* parity, int tid, int warp, int lane) {
  constexpr int MR = (1 << LOGL) / 16, NTILE = MR / 128, SPLIT = MR * 32;  // bytes per split
  // 1. split into the three BF16 operand copies: one (m, 8-wide K half) per step
  for (int q = tid; q < 2 * MR; q += kWT) {
    int m, kh;
    if (S == 1) {  // lanes 0-7: rows 0-7 of one K half (16-byte stores to consecutive core rows)
      m = (q & 7) + ((q >> 4) << 3);
      kh = (q >> 3) & 1;
    } else {       // lanes 0-15: j = 0..15 (consecutive words of X)
      m = (q & 15) + ((q >> 5) << 4);
      kh = (q >> 4) & 1;
    }
    uint32_t h[4], md[4], l[4];
#pragma unroll
    for (int e = 0; e < 8; e += 2) {
      __nv_bfloat16 h0, m0, l0, h1, m1, l1;
      split_bf16(X[phys(stage_elem<S>(m, 8 * kh + e))], h0, m0, l0);
      split_bf16(X[phys(stage_elem<S>(m, 8 * kh + e + 1))], h1, m1, l1);
      h[e >> 1] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
      md[e >> 1] = (uint32_t)__bfloat16_as_ushort(m0) | ((uint32_t)__bfloat16_as_ushort(m1) << 16);
      l[e >> 1] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
    }
    const int off = a_off(m, 8 * kh);
    *reinterpret_cast<uint4*>(As + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(As + SPLIT + off) = make_uint4(md[0], md[1], md[2], md[3]);
    *reinterpret_cast<uint4*>(As + 2 * SPLIT + off) = make_uint4(l[0], l[1], l[2], l[3]);
  }
  // generic-proxy writes of the operands -> visible to the tensor core
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  // 2. one thread issues 3 MMAs per tile into columns 16 t .. 16 t + 15
  if (tid == 0) {
    const uint64_t bdesc = kmajor_desc(smem_u32(Bs));
#pragma unroll
    for (int t = 0; t < NTILE; ++t)
#pragma unroll
      for (int s = 0; s < 3; ++s)
        mma_bf16(tbase + 16 * t, kmajor_desc(smem_u32(As + s * SPLIT + t * 4096)), bdesc, s > 0 ? 1u : 0u);
    mma_commit(bar);
  }
  const bool done = mbar_wait_bounded(bar, *parity);
  if (__syncthreads_or(!done)) return false;
  *parity ^= 1u;
  tc_fence_after();
  // 3. warp w reads TMEM lanes 32 w .. 32 w + 31 of every tile
#pragma unroll
  for (int t = 0; t < NTILE; ++t) {
    float v[16];
    tmem_ld16(tbase + ((uint32_t)(32 * warp) << 16) + 16 * t, v);
    const int m = 128 * t + 32 * warp + lane;
    if (S == 1) {
      float4* p = reinterpret_cast<float4*>(X + phys(16 * m));
#pragma unroll
      for (int q = 0; q < 4; ++q) p[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) X[phys(stage_elem<2>(m, k))] = v[k];
    }
  }
  tc_fence_before();
  __syncthreads();
  return true;
}

template <int LOGL, bool TC>
__global__ void __launch_bounds__(kWT) k_wht_rows(const float* x, float* y, int64_t rows, int* timeout) {
  constexpr int L = 1 << LOGL, MR = L / 16;
  constexpr uint32_t kCols = MR / 8 < 32 ? 32 : MR / 8;  // 16 columns per 128-row tile, power of two >= 32
  extern __shared__ __align__(1024) unsigned char sm[];
  float* X = reinterpret_cast<float*>(sm);
  unsigned char* As = sm + ((phys_len(L) * 4 + 1023) & ~1023);  // 3 splits x MR x 32 bytes
  unsigned char* Bs = As + 3 * MR * 32;                           // H16, 512 bytes
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  if (TC) {
    for (int e = tid; e < 256; e += kWT) {  // B[n][k] = H16[n][k], K-major like A
      const int n = e >> 4, k = e & 15;
      *reinterpret_cast<__nv_bfloat16*>(Bs + a_off(n, k)) = __float2bfloat16_rn((__popc(n & k) & 1) ? -1.f : 1.f);
    }
    if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                   "r"(kCols)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar)), "r"(1) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  const uint32_t tbase = TC ? tmem_base : 0u;
  uint32_t parity = 0;
  bool ok = true;
  for (int64_t r = blockIdx.x; r < rows && ok; r += gridDim.x) {
    const float4* src = reinterpret_cast<const float4*>(x + r * L);
    for (int e = tid; e < L / 4; e += kWT) *reinterpret_cast<float4*>(X + phys(4 * e)) = src[e];
    __syncthreads();
    if (TC) {
      ok = tc_stage16<LOGL, 1>(X, As, Bs, tbase, &bar, &parity, tid, warp, lane);
      if (ok) ok = tc_stage16<LOGL, 2>(X, As, Bs, tbase, &bar, &parity, tid, warp, lane);
      if (!ok) break;
    } else {
      cc_stage16<LOGL, 1>(X, tid);
      __syncthreads();
      cc_stage16<LOGL, 2>(X, tid);
      __syncthreads();
    }
    cc_stage_hi<LOGL>(X, tid);
    __syncthreads();
    float4* dst = reinterpret_cast<float4*>(y + r * L);
    for (int e = tid; e < L / 4; e += kWT) dst[e] = *reinterpret_cast<const float4*>(X + phys(4 * e));
    __syncthreads();
  }
  if (TC) {
    if (!ok) {
      if (tid == 0) atomicExch(timeout, 1);
      mbar_wait_bounded(&bar, parity);  // the MMAs this CTA issued, before their columns are freed
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
    }
    tc_fence_after();  // every warp's TMEM reads are ordered before the free (barriers above)
    if (warp == 0)
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kCols) : "memory");
  }
}

template <int LOGL, bool TC>
size_t wht_smem() {
  constexpr int L = 1 << LOGL, MR = L / 16;
  const size_t xb = ((size_t)phys_len(L) * 4 + 1023) & ~(size_t)1023;
  return TC ? xb + 3 * MR * 32 + 512 : (size_t)phys_len(L) * 4;
}

template <int LOGL, bool TC>
void wht_launch(const float* x, float* y, int64_t rows, int* timeout, cudaStream_t s) {
  const size_t smem = wht_smem<LOGL, TC>();
  // kernel attribute and resident CTAs per SM, set up once per device
  constexpr int kMaxDev = 64;
  static std::mutex mu;
  static int per_sm[kMaxDev] = {};
  int dev = 0, occ = 0;
  CMM_CUDA(cudaGetDevice(&dev));
  if (dev >= kMaxDev) throw unsupported("device index beyond 63");
  {
    std::lock_guard<std::mutex> g(mu);
    if (!per_sm[dev]) {
      CMM_CUDA(cudaFuncSetAttribute(k_wht_rows<LOGL, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      CMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_wht_rows<LOGL, TC>, kWT, smem));
      per_sm[dev] = occ < 1 ? 1 : occ;
    }
    occ = per_sm[dev];
  }
  const int64_t grid = std::min<int64_t>(rows, (int64_t)num_sms() * occ);
  k_wht_rows<LOGL, TC><<<(unsigned)grid, kWT, smem, s>>>(x, y, rows, timeout);
  CMM_CUDA(cudaGetLastError());
  count_launch();
}

// host-mapped timeout flag of the calling host thread (one per thread, so
// that concurrent calls from several threads do not clear each other's report)
int* wht_timeout_flag(int** dev) {
  thread_local int* host = nullptr;
  thread_local int* mapped = nullptr;
  if (!host) {
    int* h = nullptr;
    int* m = nullptr;
    CMM_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&h), sizeof(int), cudaHostAllocMapped));
    *h = 0;
    if (cudaHostGetDevicePointer(reinterpret_cast<void**>(&m), h, 0) != cudaSuccess) {
      cudaFreeHost(h);
      throw cuda_error("cudaHostGetDevicePointer failed for the WHT timeout flag");
    }
    host = h;  // both set only once both calls succeeded
    mapped = m;
  }
  if (dev) *dev = mapped;
  return host;
}

}  // namespace

void wht_rows_f32(const float* x, float* y, int64_t rows, int log2n, int method, cudaStream_t s) {
  if (rows < 0) throw invalid_argument("rows must be non-negative");
  if (log2n < 11 || log2n > 13) throw unsupported("the row length must be 2^11, 2^12 or 2^13");
  if (method != 0 && method != 1) throw invalid_argument("method must be 0 (CUDA cores) or 1 (tensor cores)");
  if (rows == 0) return;
  if (!x || !y) throw invalid_argument("x and y must not be null");
  if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15)
    throw invalid_argument("x and y must be 16-byte aligned");
  int* dflag = nullptr;
  volatile int* hflag = wht_timeout_flag(&dflag);
  *hflag = 0;
  const bool tc = method == 1;
  switch (log2n) {
    case 11: tc ? wht_launch<11, true>(x, y, rows, dflag, s) : wht_launch<11, false>(x, y, rows, dflag, s); break;
    case 12: tc ? wht_launch<12, true>(x, y, rows, dflag, s) : wht_launch<12, false>(x, y, rows, dflag, s); break;
    default: tc ? wht_launch<13, true>(x, y, rows, dflag, s) : wht_launch<13, false>(x, y, rows, dflag, s); break;
  }
  CMM_CUDA(cudaStreamSynchronize(s));
  if (tc) {
    if (*hflag) {
      *hflag = 0;
      throw runtime_error("tensor-core WHT: an MMA completion wait ran out");
    }
  }
}

}  // namespace cmm
