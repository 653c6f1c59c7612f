// Recovery kernels: median decompression (matmul_fft.hpp:135-147,165-177;
// matmul_fwht.hpp:122-134,154-166; array.hpp:323-328), device top-K, and
// the exact FP64 GEMM behind `gemm` (array.hpp:85-95).
#include <cfloat>

#include "cmm_internal.h"

namespace cmm {

// ------------------------------------------------------------ decompress
// Estimate for one (i, j): value_t = s1_t(i) s2_t(j) p_t[idx], idx =
// (h1+h2) & (b-1) (FFT) or h1 ^ h2 (FWHT).  With codes c = h | (s>0)<<31:
// (c1 + c2) & mask == (h1 + h2) & mask because mask < 2^31, and the product
// of the signs is negative iff bit 31 of c1 ^ c2 is set.  The sign is
// applied by flipping the sign bit, which is exactly (-1) * p.
template <int VARIANT>
__device__ __forceinline__ double estimate(const double* __restrict__ pt, uint32_t c1, uint32_t c2,
                                           uint32_t mask) {
  const uint32_t idx = VARIANT == kVariantFFT ? ((c1 + c2) & mask) : ((c1 ^ c2) & mask);
  long long bits = __double_as_longlong(__ldg(pt + idx));
  bits ^= (long long)((c1 ^ c2) & 0x80000000u) << 32;
  return __longlong_as_double(bits);
}

// sorting network by odd-even transposition; returns element D/2 of the
// ascending order (the reference's nth_element at size/2)
template <int D>
__device__ __forceinline__ double median_of(double (&v)[D]) {
#pragma unroll
  for (int pass = 0; pass < D; ++pass) {
#pragma unroll
    for (int i = pass & 1; i + 1 < D; i += 2) {
      const double lo = fmin(v[i], v[i + 1]);
      const double hi = fmax(v[i], v[i + 1]);
      v[i] = lo;
      v[i + 1] = hi;
    }
  }
  return v[D / 2];
}

constexpr int kDecThreads = 256;
constexpr int kDecRows = 16;

template <int VARIANT, int D>
__global__ void __launch_bounds__(kDecThreads) k_decompress(const uint32_t* __restrict__ cA,
                                                            const uint32_t* __restrict__ cB,
                                                            const double* __restrict__ p, int b,
                                                            int64_t n_a, int64_t n_b, int64_t lda,
                                                            double* __restrict__ C) {
  __shared__ uint32_t sA[D][kDecRows];
  const int64_t j = (int64_t)blockIdx.x * kDecThreads + threadIdx.x;
  const int64_t i0 = (int64_t)blockIdx.y * kDecRows;
  for (int e = threadIdx.x; e < D * kDecRows; e += kDecThreads) {
    const int t = e / kDecRows, ii = e % kDecRows;
    sA[t][ii] = (i0 + ii < n_a) ? cA[(size_t)t * lda + i0 + ii] : 0u;
  }
  __syncthreads();
  if (j >= n_b) return;
  uint32_t c2[D];
#pragma unroll
  for (int t = 0; t < D; ++t) c2[t] = __ldg(cB + (size_t)t * n_b + j);
  const uint32_t mask = (uint32_t)b - 1u;
  const int rows = (int)((n_a - i0) < kDecRows ? (n_a - i0) : kDecRows);
  for (int ii = 0; ii < rows; ++ii) {
    double v[D];
#pragma unroll
    for (int t = 0; t < D; ++t) v[t] = estimate<VARIANT>(p + (size_t)t * b, sA[t][ii], c2[t], mask);
    C[(size_t)(i0 + ii) * n_b + j] = median_of<D>(v);
  }
}

// any d: rank selection (element with lt <= d/2 < le), O(d^2) gathers
template <int VARIANT>
__global__ void k_decompress_generic(const uint32_t* __restrict__ cA, const uint32_t* __restrict__ cB,
                                     const double* __restrict__ p, int d, int b, int64_t n_a,
                                     int64_t n_b, int64_t lda, double* __restrict__ C) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = blockIdx.y;
  if (j >= n_b || i >= n_a) return;
  const uint32_t mask = (uint32_t)b - 1u;
  const int mid = d / 2;
  double ans = 0.0;
  for (int a = 0; a < d; ++a) {
    const double va = estimate<VARIANT>(p + (size_t)a * b, cA[(size_t)a * lda + i], cB[(size_t)a * n_b + j], mask);
    int lt = 0, le = 0;
    for (int t = 0; t < d; ++t) {
      const double vt = estimate<VARIANT>(p + (size_t)t * b, cA[(size_t)t * lda + i], cB[(size_t)t * n_b + j], mask);
      lt += vt < va;
      le += vt <= va;
    }
    if (lt <= mid && mid < le) { ans = va; break; }
  }
  C[(size_t)i * n_b + j] = ans;
}

template <int VARIANT, int D>
static void dec_launch(const uint32_t* cA, const uint32_t* cB, const double* p, int b, int64_t n_a,
                       int64_t n_b, int64_t lda, double* C, cudaStream_t s) {
  dim3 grid((unsigned)((n_b + kDecThreads - 1) / kDecThreads), (unsigned)((n_a + kDecRows - 1) / kDecRows));
  k_decompress<VARIANT, D><<<grid, kDecThreads, 0, s>>>(cA, cB, p, b, n_a, n_b, lda, C);
}

template <int VARIANT>
static void dec_dispatch(int d, const uint32_t* cA, const uint32_t* cB, const double* p, int b,
                         int64_t n_a, int64_t n_b, int64_t lda, double* C, cudaStream_t s) {
  switch (d) {
#define CMM_DEC_CASE(D) case D: dec_launch<VARIANT, D>(cA, cB, p, b, n_a, n_b, lda, C, s); return;
    CMM_DEC_CASE(1) CMM_DEC_CASE(2) CMM_DEC_CASE(3) CMM_DEC_CASE(4) CMM_DEC_CASE(5)
    CMM_DEC_CASE(6) CMM_DEC_CASE(7) CMM_DEC_CASE(8) CMM_DEC_CASE(9) CMM_DEC_CASE(10)
    CMM_DEC_CASE(11) CMM_DEC_CASE(12) CMM_DEC_CASE(13) CMM_DEC_CASE(14) CMM_DEC_CASE(15)
    CMM_DEC_CASE(16)
#undef CMM_DEC_CASE
    default: {
      if (n_a > 2147483647LL) throw unsupported("n_a too large for the generic-d decompression");
      dim3 grid((unsigned)((n_b + 255) / 256), (unsigned)n_a);
      k_decompress_generic<VARIANT><<<grid, 256, 0, s>>>(cA, cB, p, d, b, n_a, n_b, lda, C);
    }
  }
}

void launch_decompress_dense(int variant, int d, int b, int64_t n_a, int64_t n_b,
                             const uint32_t* dCodesA, const uint32_t* dCodesB, const double* dP,
                             double* dC, cudaStream_t s) {
  if (n_a <= 0 || n_b <= 0) return;
  if ((n_a + kDecRows - 1) / kDecRows > 2147483647LL) throw unsupported("n_a too large");
  ProfScope prof("decompress", s);
  count_launch();
  if (variant == kVariantFFT) dec_dispatch<kVariantFFT>(d, dCodesA, dCodesB, dP, b, n_a, n_b, n_a, dC, s);
  else dec_dispatch<kVariantFWHT>(d, dCodesA, dCodesB, dP, b, n_a, n_b, n_a, dC, s);
  CMM_CUDA(cudaGetLastError());
}

// rows [i0, i0 + rows) of the dense estimate into dCrows (rows x n_b)
void launch_decompress_dense_rows(int variant, int d, int b, int64_t n_a, int64_t n_b, int64_t i0,
                                  int64_t rows, const uint32_t* dCodesA, const uint32_t* dCodesB,
                                  const double* dP, double* dCrows, cudaStream_t s) {
  if (rows <= 0 || n_b <= 0) return;
  if (i0 < 0 || i0 + rows > n_a) throw invalid_argument("decompression rows out of range");
  if ((rows + kDecRows - 1) / kDecRows > 2147483647LL) throw unsupported("n_a too large");
  ProfScope prof("decompress", s);
  count_launch();
  if (variant == kVariantFFT) dec_dispatch<kVariantFFT>(d, dCodesA + i0, dCodesB, dP, b, rows, n_b, n_a, dCrows, s);
  else dec_dispatch<kVariantFWHT>(d, dCodesA + i0, dCodesB, dP, b, rows, n_b, n_a, dCrows, s);
  CMM_CUDA(cudaGetLastError());
}

// list form: codes are d x count, one column per listed entry
template <int VARIANT>
__global__ void k_decompress_list(const uint32_t* __restrict__ cI, const uint32_t* __restrict__ cJ,
                                  const double* __restrict__ p, int d, int b, int64_t count,
                                  double* __restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  const uint32_t mask = (uint32_t)b - 1u;
  const int mid = d / 2;
  double ans = 0.0;
  for (int a = 0; a < d; ++a) {
    const double va = estimate<VARIANT>(p + (size_t)a * b, cI[(size_t)a * count + e], cJ[(size_t)a * count + e], mask);
    int lt = 0, le = 0;
    for (int t = 0; t < d; ++t) {
      const double vt = estimate<VARIANT>(p + (size_t)t * b, cI[(size_t)t * count + e], cJ[(size_t)t * count + e], mask);
      lt += vt < va;
      le += vt <= va;
    }
    if (lt <= mid && mid < le) { ans = va; break; }
  }
  out[e] = ans;
}

void launch_decompress_list(int variant, int d, int b, int64_t count, const uint32_t* dCodesI,
                            const uint32_t* dCodesJ, const double* dP, double* dOut,
                            cudaStream_t s) {
  if (count <= 0) return;
  const unsigned blocks = (unsigned)((count + 255) / 256);
  ProfScope prof("decompress", s);
  count_launch();
  if (variant == kVariantFFT) k_decompress_list<kVariantFFT><<<blocks, 256, 0, s>>>(dCodesI, dCodesJ, dP, d, b, count, dOut);
  else k_decompress_list<kVariantFWHT><<<blocks, 256, 0, s>>>(dCodesI, dCodesJ, dP, d, b, count, dOut);
  CMM_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------ top-K
// Order-preserving 64-bit key of a double (larger key <=> larger value;
// -0.0 sorts just below +0.0, NaN with the sign bit clear above +inf).
__device__ __forceinline__ uint64_t okey(double v) {
  const uint64_t b = (uint64_t)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}

constexpr int kHistBits = 11;
constexpr int kHistBins = 1 << kHistBits;
constexpr int kLevels = 6;  // 5 x 11 bits + 9 bits = 64
constexpr int kCandMax = 4096;

__host__ __device__ __forceinline__ int digit_bits(int level) {
  return 64 - kHistBits * level < kHistBits ? 64 - kHistBits * level : kHistBits;
}

// histogram of digit `level` of the keys whose higher bits (the first
// kHistBits * level) equal `prefix`
__global__ void k_topk_hist(const double* __restrict__ C, int64_t n, int level, uint64_t prefix,
                            unsigned long long* __restrict__ hist) {
  __shared__ unsigned int sh[kHistBins];
  for (int i = threadIdx.x; i < kHistBins; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const int w = digit_bits(level);
  const int pbits = kHistBits * level;
  const int shift = 64 - pbits - w;
  const uint64_t dmask = (1ULL << w) - 1ULL;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = okey(__ldg(C + idx));
    const bool in = level == 0 || (k >> (64 - pbits)) == prefix;
    // warp-aggregated: one shared atomic per distinct digit in the warp
    // (values cluster in few digits, plain atomics would serialise)
    const uint32_t dg = in ? (uint32_t)((k >> shift) & dmask) : 0xffffffffu;
    const uint32_t active = __activemask();
    const uint32_t peers = __match_any_sync(active, dg);
    const int lane = threadIdx.x & 31;
    if (in && lane == __ffs(peers) - 1) atomicAdd(&sh[dg], (unsigned)__popc(peers));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kHistBins; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], (unsigned long long)sh[i]);
}

// one thread: walk the histogram from the top and pick the digit where the
// running count reaches `need`; out = {digit, count_above_in_level, count_in_bin}
__global__ void k_topk_pick(const unsigned long long* __restrict__ hist, int nbins,
                            unsigned long long need, unsigned long long* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long run = 0;
  for (int dgt = nbins - 1; dgt >= 0; --dgt) {
    const unsigned long long c = hist[dgt];
    if (run + c >= need) {
      out[0] = (unsigned long long)dgt;
      out[1] = run;
      out[2] = c;
      return;
    }
    run += c;
  }
  out[0] = 0; out[1] = run; out[2] = 0;
}

// collect entries whose key prefix (top `pbits` bits) is >= pfx (strictly
// greater if `strict`) into the candidate buffer
__global__ void k_topk_collect(const double* __restrict__ C, int64_t n, int pbits, uint64_t pfx,
                               int strict, unsigned long long* __restrict__ keys,
                               unsigned long long* __restrict__ idxs, unsigned int* __restrict__ count,
                               unsigned int cap) {
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = okey(__ldg(C + idx));
    const uint64_t top = pbits >= 64 ? k : (k >> (64 - pbits));
    if (strict ? top > pfx : top >= pfx) {
      const unsigned int slot = atomicAdd(count, 1u);
      if (slot < cap) { keys[slot] = k; idxs[slot] = (unsigned long long)idx; }
    }
  }
}

// ordered collection of the first `need` entries equal to key `tau`
// (ties broken by linear index = (i, j) order): per-block counts, then
// block-ordered writes.
__global__ void k_topk_tie_count(const double* __restrict__ C, int64_t n, uint64_t tau,
                                 int64_t chunk, unsigned long long* __restrict__ counts) {
  const int64_t beg = (int64_t)blockIdx.x * chunk;
  const int64_t end = beg + chunk < n ? beg + chunk : n;
  unsigned long long c = 0;
  for (int64_t idx = beg + threadIdx.x; idx < end; idx += blockDim.x) c += okey(__ldg(C + idx)) == tau;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  __shared__ unsigned long long s[32];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += s[w];
    counts[blockIdx.x] = tot;
  }
}

__global__ void k_topk_tie_write(const double* __restrict__ C, int64_t n, uint64_t tau, int64_t chunk,
                                 const unsigned long long* __restrict__ counts, int nblocks,
                                 unsigned long long need, unsigned long long* __restrict__ keys,
                                 unsigned long long* __restrict__ idxs, unsigned int base) {
  // serial within the block, in index order (only blocks that contribute)
  if (threadIdx.x != 0) return;
  unsigned long long before = 0;
  for (int blk = 0; blk < (int)blockIdx.x; ++blk) before += counts[blk];
  if (before >= need || counts[blockIdx.x] == 0) return;
  const int64_t beg = (int64_t)blockIdx.x * chunk;
  const int64_t end = beg + chunk < n ? beg + chunk : n;
  unsigned long long r = before;
  for (int64_t idx = beg; idx < end && r < need; ++idx) {
    if (okey(C[idx]) == tau) {
      keys[base + r] = tau;
      idxs[base + r] = (unsigned long long)idx;
      ++r;
    }
  }
}

// single-CTA bitonic sort of up to kCandMax candidates: key descending,
// index ascending; writes the first K as (i, j, value)
__global__ void __launch_bounds__(1024) k_topk_sort(const unsigned long long* __restrict__ keys,
                                                     const unsigned long long* __restrict__ idxs,
                                                     const unsigned int* __restrict__ count,
                                                     int K, int64_t n_b, uint32_t* oi, uint32_t* oj,
                                                     double* ov) {
  extern __shared__ unsigned long long sdyn[];
  unsigned long long* sk = sdyn;
  unsigned long long* si = sdyn + kCandMax;
  const unsigned int n = *count < (unsigned)kCandMax ? *count : (unsigned)kCandMax;
  for (int e = threadIdx.x; e < kCandMax; e += blockDim.x) {
    if ((unsigned)e < n) { sk[e] = keys[e]; si[e] = idxs[e]; }
    else { sk[e] = 0ULL; si[e] = ~0ULL; }
  }
  __syncthreads();
  // "a before b" := key_a > key_b || (key_a == key_b && idx_a < idx_b)
  for (int size = 2; size <= kCandMax; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int e = threadIdx.x; e < kCandMax; e += blockDim.x) {
        const int partner = e ^ stride;
        if (partner > e) {
          const bool asc = (e & size) == 0;  // first half of each block: "before" order
          const unsigned long long ka = sk[e], kb = sk[partner];
          const unsigned long long ia = si[e], ib = si[partner];
          const bool b_before_a = (kb > ka) || (kb == ka && ib < ia);
          if (asc ? b_before_a : !b_before_a) {
            sk[e] = kb; sk[partner] = ka;
            si[e] = ib; si[partner] = ia;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int e = threadIdx.x; e < K; e += blockDim.x) {
    const unsigned long long key = sk[e];
    const unsigned long long bits = (key >> 63) ? (key & 0x7fffffffffffffffULL) : ~key;
    const unsigned long long id = si[e];
    oi[e] = (uint32_t)(id / (unsigned long long)n_b);
    oj[e] = (uint32_t)(id % (unsigned long long)n_b);
    ov[e] = __longlong_as_double((long long)bits);
  }
}

void topk_dense(const double* dC, int64_t n_a, int64_t n_b, int K, uint32_t* dI, uint32_t* dJ,
                double* dV, cudaStream_t s) {
  const int64_t n = n_a * n_b;
  if (K <= 0) return;
  if (K > kCandMax) throw unsupported("K > 4096 is not supported by the device top-K");
  if ((int64_t)K > n) throw invalid_argument("K exceeds the number of entries");
  ProfScope prof("topk", s);
  DevBuf hist((size_t)kHistBins * 8, s), pick(3 * 8, s);
  DevBuf keys((size_t)kCandMax * 8, s), idxs((size_t)kCandMax * 8, s), cnt(8, s);
  int64_t blocks = (n + 255) / 256;
  if (blocks > 4 * num_sms()) blocks = 4 * num_sms();
  uint64_t prefix = 0;              // selected digits so far
  unsigned long long need = (unsigned long long)K;  // still to take at this prefix
  unsigned long long above = 0;     // taken strictly above the prefix (all levels)
  int level = 0;
  int pbits = 0;
  unsigned long long h_pick[3];
  bool tie = false;
  for (; level < kLevels; ++level) {
    const int w = digit_bits(level);
    CMM_CUDA(cudaMemsetAsync(hist.ptr, 0, hist.bytes, s));
    count_launch(2);
    k_topk_hist<<<(unsigned)blocks, 256, 0, s>>>(dC, n, level, prefix, hist.as<unsigned long long>());
    CMM_CUDA(cudaGetLastError());
    k_topk_pick<<<1, 32, 0, s>>>(hist.as<unsigned long long>(), 1 << w, need,
                                 pick.as<unsigned long long>());
    CMM_CUDA(cudaMemcpyAsync(h_pick, pick.ptr, sizeof(h_pick), cudaMemcpyDeviceToHost, s));
    CMM_CUDA(cudaStreamSynchronize(s));
    prefix = (prefix << w) | h_pick[0];
    pbits += w;
    above += h_pick[1];
    need -= h_pick[1];
    // everything at this prefix fits: collect >= prefix and sort
    if (above + h_pick[2] <= (unsigned long long)kCandMax) break;
    if (level == kLevels - 1) tie = true;  // > kCandMax entries share the K-th key exactly
  }
  CMM_CUDA(cudaMemsetAsync(cnt.ptr, 0, 8, s));
  count_launch(tie ? 4 : 2);
  if (!tie) {
    k_topk_collect<<<(unsigned)blocks, 256, 0, s>>>(dC, n, pbits, prefix, 0, keys.as<unsigned long long>(),
                                                    idxs.as<unsigned long long>(), cnt.as<unsigned int>(), kCandMax);
    CMM_CUDA(cudaGetLastError());
  } else {
    // strictly greater keys (< K of them), then the first `need` ties by index
    k_topk_collect<<<(unsigned)blocks, 256, 0, s>>>(dC, n, 64, prefix, 1, keys.as<unsigned long long>(),
                                                    idxs.as<unsigned long long>(), cnt.as<unsigned int>(), kCandMax);
    CMM_CUDA(cudaGetLastError());
    const int64_t chunk = 1 << 20;
    const int nb = (int)((n + chunk - 1) / chunk);
    DevBuf counts((size_t)nb * 8, s);
    k_topk_tie_count<<<nb, 256, 0, s>>>(dC, n, prefix, chunk, counts.as<unsigned long long>());
    k_topk_tie_write<<<nb, 32, 0, s>>>(dC, n, prefix, chunk, counts.as<unsigned long long>(), nb, need,
                                       keys.as<unsigned long long>(), idxs.as<unsigned long long>(),
                                       (unsigned int)above);
    CMM_CUDA(cudaGetLastError());
    const unsigned int total = (unsigned int)K;
    CMM_CUDA(cudaMemcpyAsync(cnt.ptr, &total, 4, cudaMemcpyHostToDevice, s));
  }
  const int ssmem = 2 * kCandMax * 8;
  CMM_CUDA(cudaFuncSetAttribute(k_topk_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, ssmem));
  k_topk_sort<<<1, 1024, ssmem, s>>>(keys.as<unsigned long long>(), idxs.as<unsigned long long>(),
                                  cnt.as<unsigned int>(), K, n_b, dI, dJ, dV);
  CMM_CUDA(cudaGetLastError());
  CMM_CUDA(cudaStreamSynchronize(s));
}

// ------------------------------------------------------------------- GEMM
// C[i][j] = sum_k AT[k][i] B[k][j]; 64x64 tiles, 16-deep k slabs, 4x4 per
// thread, FP64 FMA.
constexpr int kGT = 64, kGK = 16;
__global__ void __launch_bounds__(256) k_gemm(const double* __restrict__ AT, const double* __restrict__ B,
                                              int64_t n_a, int64_t n_inner, int64_t n_b,
                                              double* __restrict__ C) {
  __shared__ double As[kGK][kGT];
  __shared__ double Bs[kGK][kGT];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t i0 = (int64_t)blockIdx.y * kGT, j0 = (int64_t)blockIdx.x * kGT;
  double acc[4][4] = {};
  for (int64_t k0 = 0; k0 < n_inner; k0 += kGK) {
    for (int e = threadIdx.x; e < kGK * kGT; e += 256) {
      const int kk = e / kGT, c = e % kGT;
      const int64_t k = k0 + kk;
      As[kk][c] = (k < n_inner && i0 + c < n_a) ? AT[k * n_a + i0 + c] : 0.0;
      Bs[kk][c] = (k < n_inner && j0 + c < n_b) ? B[k * n_b + j0 + c] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGK; ++kk) {
      double a[4], bb[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { a[u] = As[kk][ty + 16 * u]; bb[u] = Bs[kk][tx + 16 * u]; }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], bb[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int64_t i = i0 + ty + 16 * u, j = j0 + tx + 16 * v;
      if (i < n_a && j < n_b) C[i * n_b + j] = acc[u][v];
    }
}

void launch_gemm(int64_t n_a, int64_t n_inner, int64_t n_b, double* dC, const double* dAT,
                 const double* dB, cudaStream_t s) {
  if (n_a <= 0 || n_b <= 0) return;
  if (n_inner <= 0) {
    CMM_CUDA(cudaMemsetAsync(dC, 0, (size_t)n_a * n_b * sizeof(double), s));
    return;
  }
  dim3 grid((unsigned)((n_b + kGT - 1) / kGT), (unsigned)((n_a + kGT - 1) / kGT));
  ProfScope prof("gemm", s);
  count_launch();
  k_gemm<<<grid, 256, 0, s>>>(dAT, dB, n_a, n_inner, n_b, dC);
  CMM_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------- conversion
__global__ void k_f32_to_f64(const float* __restrict__ src, double* __restrict__ dst, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

void launch_f32_to_f64(const float* src, double* dst, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  int64_t blocks = (n + 255) / 256;
  if (blocks > 8 * num_sms()) blocks = 8 * num_sms();
  count_launch();
  k_f32_to_f64<<<(unsigned)blocks, 256, 0, s>>>(src, dst, n);
  CMM_CUDA(cudaGetLastError());
}

}  // namespace cmm
