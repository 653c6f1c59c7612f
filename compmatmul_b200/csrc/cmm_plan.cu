// Sketch plans: the per-call, data-independent layout that turns the count
// sketch into conflict-free register accumulation.
//
// For each repetition t and side (A: h1/s1 over i < n_a, B: h2/s2 over
// j < n_b) the indices are stably sorted by n = h mod L (their bucket inside
// one transform slab).  The sorted list is cut into kPlanThreads contiguous
// ranges at bucket boundaries, one per thread of the sketch kernel, so every
// bucket has exactly one owner thread.  Slot (s, j) = s * kPlanThreads + j
// holds the s-th index of thread j's range: consecutive threads read
// consecutive slots (coalesced), and each thread sees its buckets in
// non-decreasing order (runs accumulate in registers, one store per bucket).
//
// The plan depends only on (hash functions, n_a, n_b, L); the matrices are
// then "materialized" per t in slot order with the sign applied, in chunks
// of inner indices (k_materialize), and read by the sketch kernels.
#include "cmm_internal.h"

namespace cmm {

constexpr int kSortThreads = 1024;

// Stable counting sort of one (t, side) by n = code & (L-1); outputs the
// sorted index list, the cut points of the kPlanThreads ranges and the
// largest range.  grid (d, 2), dynamic smem (L + 1) * 4 * 2 bytes.
__global__ void __launch_bounds__(kSortThreads) k_plan_sort(const uint32_t* __restrict__ codesA,
                                                           const uint32_t* __restrict__ codesB,
                                                           int64_t n_a, int64_t n_b, int logL,
                                                           uint32_t* __restrict__ sortedA,
                                                           uint32_t* __restrict__ sortedB,
                                                           uint32_t* __restrict__ cut,
                                                           uint32_t* __restrict__ emax) {
  extern __shared__ uint32_t ssort[];
  const int L = 1 << logL;
  uint32_t* cnt = ssort;          // L + 1: running positions
  uint32_t* cum = ssort + L + 1;  // L + 1: bucket starts
  const int t = blockIdx.x, side = blockIdx.y;
  const int64_t N = side == 0 ? n_a : n_b;
  const uint32_t* codes = (side == 0 ? codesA : codesB) + (size_t)t * N;
  uint32_t* sorted = (side == 0 ? sortedA : sortedB) + (size_t)t * N;
  const uint32_t mask = (uint32_t)L - 1u;
  for (int e = threadIdx.x; e <= L; e += kSortThreads) cnt[e] = 0;
  __syncthreads();
  for (int64_t i = threadIdx.x; i < N; i += kSortThreads) atomicAdd(&cnt[__ldg(codes + i) & mask], 1u);
  __syncthreads();
  // exclusive scan of cnt[0..L) into cum (single warp, L <= 2^14)
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const int per = (L + 31) / 32;
    uint32_t local = 0;
    for (int e = lane * per; e < (lane + 1) * per && e < L; ++e) local += cnt[e];
    uint32_t incl = local;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    uint32_t run = incl - local;
    for (int e = lane * per; e < (lane + 1) * per && e < L; ++e) {
      const uint32_t c = cnt[e];
      cum[e] = run;
      run += c;
    }
    if (lane == 31) cum[L] = incl;
  }
  __syncthreads();
  for (int e = threadIdx.x; e <= L; e += kSortThreads) cnt[e] = cum[e];
  __syncthreads();
  // stable placement, one warp at a time within each tile of 1024 indices
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t base = 0; base < N; base += kSortThreads) {
    const int64_t i = base + threadIdx.x;
    const bool valid = i < N;
    const uint32_t key = valid ? (__ldg(codes + i) & mask) : (0x80000000u | (uint32_t)lane);
    const uint32_t peers = __match_any_sync(0xffffffffu, key);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    for (int w = 0; w < kSortThreads / 32; ++w) {
      if (warp == w && valid) {
        const uint32_t pos = cnt[key] + rank;
        sorted[pos] = (uint32_t)i;
      }
      __syncwarp();
      if (warp == w && valid && rank == 0) cnt[key] += __popc(peers);
      __syncthreads();
    }
  }
  // cut points: thread j of the sketch kernel starts at bucket B_j = first
  // bucket whose start >= j * N / T; cut[j] = cum[B_j] (an index position)
  uint32_t* cuts = cut + ((size_t)t * 2 + side) * (kPlanThreads + 1);
  for (int j = threadIdx.x; j <= kPlanThreads; j += kSortThreads) {
    const uint64_t target = ((uint64_t)j * (uint64_t)N) / kPlanThreads;
    int lo = 0, hi = L;  // smallest b in [0, L] with cum[b] >= target
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (cum[mid] >= target) hi = mid;
      else lo = mid + 1;
    }
    cuts[j] = j == kPlanThreads ? (uint32_t)N : cum[lo];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t m = 0;
    for (int j = 0; j < kPlanThreads; ++j) {
      const uint32_t c = cuts[j + 1] - cuts[j];
      m = c > m ? c : m;
    }
    emax[t * 2 + side] = m;
  }
}

// slot arrays of one (t, side): src = index | (sign == +1) << 31 (or
// kPadSlot), code = bucket h (u16 when b <= 2^16, else u32), count per thread
template <typename CodeT>
__global__ void k_plan_layout(const uint32_t* __restrict__ codesA, const uint32_t* __restrict__ codesB,
                              int64_t n_a, int64_t n_b, const uint32_t* __restrict__ sortedA,
                              const uint32_t* __restrict__ sortedB, const uint32_t* __restrict__ cut,
                              int EA, int EB, uint32_t* __restrict__ srcA, uint32_t* __restrict__ srcB,
                              CodeT* __restrict__ codeA, CodeT* __restrict__ codeB,
                              uint32_t* __restrict__ countA, uint32_t* __restrict__ countB) {
  const int t = blockIdx.y, side = blockIdx.z;
  const int E = side == 0 ? EA : EB;
  const int64_t N = side == 0 ? n_a : n_b;
  const uint32_t* codes = (side == 0 ? codesA : codesB) + (size_t)t * N;
  const uint32_t* sorted = (side == 0 ? sortedA : sortedB) + (size_t)t * N;
  const uint32_t* cuts = cut + ((size_t)t * 2 + side) * (kPlanThreads + 1);
  const size_t S = (size_t)E * kPlanThreads;
  uint32_t* src = (side == 0 ? srcA : srcB) + (size_t)t * S;
  CodeT* code = (side == 0 ? codeA : codeB) + (size_t)t * S;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)S;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(e % kPlanThreads);
    const uint32_t s = (uint32_t)(e / kPlanThreads);
    const uint32_t beg = cuts[j], end = cuts[j + 1];
    if (beg + s < end) {
      const uint32_t i = sorted[beg + s];
      const uint32_t c = codes[i];
      src[e] = i | (c & 0x80000000u);
      code[e] = (CodeT)(c & 0x7fffffffu);
    } else {
      src[e] = kPadSlot;
      code[e] = 0;
    }
  }
  if (blockIdx.x == 0)
    for (int j = threadIdx.x; j < kPlanThreads; j += blockDim.x)
      (side == 0 ? countA : countB)[(size_t)t * kPlanThreads + j] = cuts[j + 1] - cuts[j];
}

SlabPlan make_slab_plan(const uint32_t* dCodesA, const uint32_t* dCodesB, int64_t n_a, int64_t n_b,
                        int d, int b, int logL, cudaStream_t s) {
  SlabPlan P;
  P.d = d;
  P.logL = logL;
  P.n_a = n_a;
  P.n_b = n_b;
  P.u16 = b <= 65536;
  const int L = 1 << logL;
  DevBuf sortedA((size_t)d * (n_a > 0 ? n_a : 1) * 4, s), sortedB((size_t)d * (n_b > 0 ? n_b : 1) * 4, s);
  DevBuf cut((size_t)d * 2 * (kPlanThreads + 1) * 4, s), emax((size_t)d * 2 * 4, s);
  const int smem = 2 * (L + 1) * 4;
  CMM_CUDA(cudaFuncSetAttribute(k_plan_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  {
    ProfScope prof("plan", s);
    count_launch();
    k_plan_sort<<<dim3(d, 2), kSortThreads, smem, s>>>(dCodesA, dCodesB, n_a, n_b, logL,
                                                       sortedA.as<uint32_t>(), sortedB.as<uint32_t>(),
                                                       cut.as<uint32_t>(), emax.as<uint32_t>());
    CMM_CUDA(cudaGetLastError());
  }
  std::vector<uint32_t> h((size_t)d * 2);
  CMM_CUDA(cudaMemcpyAsync(h.data(), emax.ptr, h.size() * 4, cudaMemcpyDeviceToHost, s));
  CMM_CUDA(cudaStreamSynchronize(s));
  P.EA = 1;
  P.EB = 1;
  for (int t = 0; t < d; ++t) {
    P.EA = (int)(h[2 * t] > (uint32_t)P.EA ? h[2 * t] : P.EA);
    P.EB = (int)(h[2 * t + 1] > (uint32_t)P.EB ? h[2 * t + 1] : P.EB);
  }
  const size_t SA = (size_t)P.EA * kPlanThreads, SB = (size_t)P.EB * kPlanThreads;
  const size_t cb = P.u16 ? 2 : 4;
  P.srcA = DevBuf((size_t)d * SA * 4, s);
  P.srcB = DevBuf((size_t)d * SB * 4, s);
  P.codeA = DevBuf((size_t)d * SA * cb, s);
  P.codeB = DevBuf((size_t)d * SB * cb, s);
  P.countA = DevBuf((size_t)d * kPlanThreads * 4, s);
  P.countB = DevBuf((size_t)d * kPlanThreads * 4, s);
  const size_t Smax = SA > SB ? SA : SB;
  dim3 grid((unsigned)((Smax + 255) / 256 < 1024 ? (Smax + 255) / 256 : 1024), (unsigned)d, 2);
  ProfScope prof("plan", s);
  count_launch();
  if (P.u16)
    k_plan_layout<uint16_t><<<grid, 256, 0, s>>>(dCodesA, dCodesB, n_a, n_b, sortedA.as<uint32_t>(),
                                                 sortedB.as<uint32_t>(), cut.as<uint32_t>(), P.EA, P.EB,
                                                 P.srcA.as<uint32_t>(), P.srcB.as<uint32_t>(),
                                                 P.codeA.as<uint16_t>(), P.codeB.as<uint16_t>(),
                                                 P.countA.as<uint32_t>(), P.countB.as<uint32_t>());
  else
    k_plan_layout<uint32_t><<<grid, 256, 0, s>>>(dCodesA, dCodesB, n_a, n_b, sortedA.as<uint32_t>(),
                                                 sortedB.as<uint32_t>(), cut.as<uint32_t>(), P.EA, P.EB,
                                                 P.srcA.as<uint32_t>(), P.srcB.as<uint32_t>(),
                                                 P.codeA.as<uint32_t>(), P.codeB.as<uint32_t>(),
                                                 P.countA.as<uint32_t>(), P.countB.as<uint32_t>());
  CMM_CUDA(cudaGetLastError());
  (void)L;
  return P;
}

// ---------------------------------------------------------- materialize
// out[t][kk][e] = sign * row_k[src[t][e]] (0 for padding), for both sides,
// for inner indices k0 + kk, kk < kc.  One CTA of 1024 threads per inner
// index; the row is staged in shared memory when it fits.  Each thread
// writes four consecutive slots (S is a multiple of 8): one 16-byte load of
// their indices, two 16-byte streaming stores (the copies are read back
// once, by the sketch kernel).
constexpr int kMatThreads = 1024;

template <bool STAGE>
__global__ void __launch_bounds__(kMatThreads) k_materialize(const double* __restrict__ AT,
                                                            const double* __restrict__ B, int64_t n_a,
                                                            int64_t n_b, int64_t k0, int d,
                                                            const uint32_t* __restrict__ srcA,
                                                            const uint32_t* __restrict__ srcB,
                                                            int64_t SA, int64_t SB, int64_t kc,
                                                            double* __restrict__ outA,
                                                            double* __restrict__ outB) {
  extern __shared__ double srow[];
  const int64_t kk = blockIdx.x;
  for (int side = 0; side < 2; ++side) {
    const int64_t N = side == 0 ? n_a : n_b;
    const int64_t S = side == 0 ? SA : SB;
    const double* row = (side == 0 ? AT : B) + (size_t)(k0 + kk) * N;
    const uint32_t* src = side == 0 ? srcA : srcB;
    double* out = side == 0 ? outA : outB;
    if (STAGE) {
      for (int64_t i = threadIdx.x; i < N; i += kMatThreads) srow[i] = __ldg(row + i);
      __syncthreads();
    }
    for (int t = 0; t < d; ++t) {
      const uint4* st = reinterpret_cast<const uint4*>(src + (size_t)t * S);
      double2* ot = reinterpret_cast<double2*>(out + ((size_t)t * kc + kk) * S);
      for (int64_t q = threadIdx.x; q < S / 4; q += kMatThreads) {
        const uint4 sv = __ldg(st + q);
        const uint32_t svs[4] = {sv.x, sv.y, sv.z, sv.w};
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          v[u] = 0.0;
          if (svs[u] != kPadSlot) {
            v[u] = STAGE ? srow[svs[u] & 0x7fffffffu] : __ldg(row + (svs[u] & 0x7fffffffu));
            if (!(svs[u] >> 31)) v[u] = -v[u];
          }
        }
        __stcs(ot + 2 * q, make_double2(v[0], v[1]));
        __stcs(ot + 2 * q + 1, make_double2(v[2], v[3]));
      }
    }
    __syncthreads();
  }
}

void launch_materialize(const SlabPlan& P, const double* dAT, const double* dB, int64_t k0,
                        int64_t kc, double* dOutA, double* dOutB, cudaStream_t s) {
  if (kc <= 0) return;
  const int64_t nmax = P.n_a > P.n_b ? P.n_a : P.n_b;
  const size_t smem = (size_t)nmax * 8;
  const int64_t SA = P.slots_a(), SB = P.slots_b();
  if (SA % 4 || SB % 4) throw runtime_error("materialize: segment slots must be a multiple of 4");
  ProfScope prof("materialize", s);
  count_launch();
  if (smem <= 200 * 1024) {
    CMM_CUDA(cudaFuncSetAttribute(k_materialize<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_materialize<true><<<(unsigned)kc, kMatThreads, smem, s>>>(dAT, dB, P.n_a, P.n_b, k0, P.d,
                                                                P.srcA.as<uint32_t>(), P.srcB.as<uint32_t>(),
                                                                SA, SB, kc, dOutA, dOutB);
  } else {
    k_materialize<false><<<(unsigned)kc, kMatThreads, 0, s>>>(dAT, dB, P.n_a, P.n_b, k0, P.d,
                                                              P.srcA.as<uint32_t>(), P.srcB.as<uint32_t>(),
                                                              SA, SB, kc, dOutA, dOutB);
  }
  CMM_CUDA(cudaGetLastError());
}

}  // namespace cmm

namespace cmm {

// ------------------------------------------------------ residue plans
// Plans for the cluster kernels (cmm_sketch_cluster.cu).  With
// b = R1 * R2 * L, an index with bucket h belongs to residue class
// r2 = h mod R2 and sub-bucket m = (h mod (b / R1)) div R2 (< L); its DIF
// quotient is q1 = h div (b / R1).  Per (t, side, r2) the members are
// stably sorted by m and cut into kPlanThreads ranges at bucket boundaries;
// slot (s, j) of segment r2 sits at [r2][s * kPlanThreads + j].  The code of
// a slot is m | q1 << logL.
constexpr int kSegSortThreads = 1024;

__global__ void __launch_bounds__(kSegSortThreads) k_plan_seg_sort(
    const uint32_t* __restrict__ codesA, const uint32_t* __restrict__ codesB, int64_t n_a, int64_t n_b,
    int logL, int logR2, int logM, uint32_t* __restrict__ sortedA, uint32_t* __restrict__ sortedB,
    uint32_t* __restrict__ cut, uint32_t* __restrict__ emax) {
  extern __shared__ uint32_t sseg[];
  const int L = 1 << logL, R2 = 1 << logR2;
  uint32_t* cnt = sseg;
  uint32_t* cum = sseg + L + 1;
  const int t = blockIdx.x, side = blockIdx.y, r2 = blockIdx.z;
  const int d2 = gridDim.z;
  const int64_t N = side == 0 ? n_a : n_b;
  const uint32_t* codes = (side == 0 ? codesA : codesB) + (size_t)t * N;
  // segment output: sorted[t][r2][0..N) holds the members of residue r2
  uint32_t* sorted = (side == 0 ? sortedA : sortedB) + ((size_t)t * d2 + r2) * N;
  const uint32_t rmask = (uint32_t)R2 - 1u, mmask = (1u << logM) - 1u;
  for (int e = threadIdx.x; e <= L; e += kSegSortThreads) cnt[e] = 0;
  __syncthreads();
  for (int64_t i = threadIdx.x; i < N; i += kSegSortThreads) {
    const uint32_t h = __ldg(codes + i) & 0x7fffffffu;
    if ((h & rmask) == (uint32_t)r2) atomicAdd(&cnt[(h & mmask) >> logR2], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const int per = (L + 31) / 32;
    uint32_t local = 0;
    for (int e = lane * per; e < (lane + 1) * per && e < L; ++e) local += cnt[e];
    uint32_t incl = local;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    uint32_t run = incl - local;
    for (int e = lane * per; e < (lane + 1) * per && e < L; ++e) {
      const uint32_t c = cnt[e];
      cum[e] = run;
      run += c;
    }
    if (lane == 31) cum[L] = incl;
  }
  __syncthreads();
  for (int e = threadIdx.x; e <= L; e += kSegSortThreads) cnt[e] = cum[e];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t base = 0; base < N; base += kSegSortThreads) {
    const int64_t i = base + threadIdx.x;
    bool valid = i < N;
    uint32_t key = 0x80000000u | (uint32_t)lane;
    if (valid) {
      const uint32_t h = __ldg(codes + i) & 0x7fffffffu;
      valid = (h & rmask) == (uint32_t)r2;
      if (valid) key = (h & mmask) >> logR2;
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, key);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    for (int w = 0; w < kSegSortThreads / 32; ++w) {
      if (warp == w && valid) sorted[cnt[key] + rank] = (uint32_t)i;
      __syncwarp();
      if (warp == w && valid && rank == 0) cnt[key] += __popc(peers);
      __syncthreads();
    }
  }
  const uint32_t total = cum[L];
  uint32_t* cuts = cut + (((size_t)t * 2 + side) * d2 + r2) * (kPlanThreads + 1);
  for (int j = threadIdx.x; j <= kPlanThreads; j += kSegSortThreads) {
    const uint64_t target = ((uint64_t)j * (uint64_t)total) / kPlanThreads;
    int lo = 0, hi = L;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (cum[mid] >= target) hi = mid;
      else lo = mid + 1;
    }
    cuts[j] = j == kPlanThreads ? total : cum[lo];
  }
  if (threadIdx.x == 0) emax[((size_t)t * 2 + side) * d2 + r2] = total;  // segment size
}

template <typename CodeT>
__global__ void k_plan_seg_layout(const uint32_t* __restrict__ codesA, const uint32_t* __restrict__ codesB,
                                  int64_t n_a, int64_t n_b, int logL, int logR2, int logM, int R2,
                                  const uint32_t* __restrict__ sortedA, const uint32_t* __restrict__ sortedB,
                                  const uint32_t* __restrict__ cut, int SA, int SB,
                                  uint32_t* __restrict__ srcA, uint32_t* __restrict__ srcB,
                                  CodeT* __restrict__ codeA, CodeT* __restrict__ codeB,
                                  uint32_t* __restrict__ cutA, uint32_t* __restrict__ cutB) {
  const int t = blockIdx.y;
  const int side = blockIdx.z & 1, r2 = blockIdx.z >> 1;
  const int S = side == 0 ? SA : SB;
  const int64_t N = side == 0 ? n_a : n_b;
  const uint32_t* codes = (side == 0 ? codesA : codesB) + (size_t)t * N;
  const uint32_t* sorted = (side == 0 ? sortedA : sortedB) + ((size_t)t * R2 + r2) * N;
  const uint32_t* cuts = cut + (((size_t)t * 2 + side) * R2 + r2) * (kPlanThreads + 1);
  const uint32_t total = cuts[kPlanThreads];
  uint32_t* src = (side == 0 ? srcA : srcB) + ((size_t)t * R2 + r2) * S;
  CodeT* code = (side == 0 ? codeA : codeB) + ((size_t)t * R2 + r2) * S;
  const uint32_t mmask = (1u << logM) - 1u;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < S; e += (int64_t)gridDim.x * blockDim.x) {
    if ((uint32_t)e < total) {
      const uint32_t i = sorted[e];
      const uint32_t c = codes[i];
      const uint32_t h = c & 0x7fffffffu;
      src[e] = i | (c & 0x80000000u);
      code[e] = (CodeT)(((h & mmask) >> logR2) | ((h >> logM) << logL));
    } else {
      src[e] = kPadSlot;
      code[e] = 0;
    }
  }
  if (blockIdx.x == 0)
    for (int j = threadIdx.x; j <= kPlanThreads; j += blockDim.x)
      (side == 0 ? cutA : cutB)[((size_t)t * R2 + r2) * (kPlanThreads + 1) + j] = cuts[j];
}

SlabPlan make_residue_plan(const uint32_t* dCodesA, const uint32_t* dCodesB, int64_t n_a, int64_t n_b,
                           int d, int b, int logL, int logR2, cudaStream_t s) {
  SlabPlan P;
  P.d = d;
  P.logL = logL;
  P.n_a = n_a;
  P.n_b = n_b;
  int log2b = 0;
  while ((1 << log2b) < b) ++log2b;
  const int logR1 = log2b - logL - logR2;
  const int logM = log2b - logR1;  // log2(b / R1)
  P.segs = 1 << logR2;
  // code = m (logL bits) | q1 << logL (logR1 bits)
  P.u16 = logL + logR1 <= 16;
  const int L = 1 << logL, R2 = 1 << logR2;
  DevBuf sortedA((size_t)d * R2 * (n_a > 0 ? n_a : 1) * 4, s), sortedB((size_t)d * R2 * (n_b > 0 ? n_b : 1) * 4, s);
  DevBuf cut((size_t)d * 2 * R2 * (kPlanThreads + 1) * 4, s), emax((size_t)d * 2 * R2 * 4, s);
  const int smem = 2 * (L + 1) * 4;
  CMM_CUDA(cudaFuncSetAttribute(k_plan_seg_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  {
    ProfScope prof("plan", s);
    count_launch();
    k_plan_seg_sort<<<dim3(d, 2, R2), kSegSortThreads, smem, s>>>(
        dCodesA, dCodesB, n_a, n_b, logL, logR2, logM, sortedA.as<uint32_t>(), sortedB.as<uint32_t>(),
        cut.as<uint32_t>(), emax.as<uint32_t>());
    CMM_CUDA(cudaGetLastError());
  }
  // compact segments: S = the largest segment (over t and r2), rounded to 8;
  // with one segment (R2 = 1) it holds every index, so no read-back is needed
  uint32_t SA = 8, SB = 8;
  if (R2 == 1) {
    SA = n_a > 8 ? (uint32_t)n_a : 8u;
    SB = n_b > 8 ? (uint32_t)n_b : 8u;
  } else {
    std::vector<uint32_t> h((size_t)d * 2 * R2);
    CMM_CUDA(cudaMemcpyAsync(h.data(), emax.ptr, h.size() * 4, cudaMemcpyDeviceToHost, s));
    CMM_CUDA(cudaStreamSynchronize(s));
    for (int t = 0; t < d; ++t)
      for (int r = 0; r < R2; ++r) {
        SA = h[((size_t)t * 2 + 0) * R2 + r] > SA ? h[((size_t)t * 2 + 0) * R2 + r] : SA;
        SB = h[((size_t)t * 2 + 1) * R2 + r] > SB ? h[((size_t)t * 2 + 1) * R2 + r] : SB;
      }
  }
  SA = (SA + 7) & ~7u;
  SB = (SB + 7) & ~7u;
  P.compact = true;
  P.EA = (int)SA;  // slots per segment (not per thread) for compact plans
  P.EB = (int)SB;
  const size_t cb = P.u16 ? 2 : 4;
  P.srcA = DevBuf((size_t)d * R2 * SA * 4, s);
  P.srcB = DevBuf((size_t)d * R2 * SB * 4, s);
  P.codeA = DevBuf((size_t)d * R2 * SA * cb, s);
  P.codeB = DevBuf((size_t)d * R2 * SB * cb, s);
  P.countA = DevBuf((size_t)d * R2 * (kPlanThreads + 1) * 4, s);
  P.countB = DevBuf((size_t)d * R2 * (kPlanThreads + 1) * 4, s);
  const size_t Smax = SA > SB ? SA : SB;
  dim3 grid((unsigned)((Smax + 255) / 256 < 256 ? (Smax + 255) / 256 : 256), (unsigned)d, (unsigned)(2 * R2));
  ProfScope prof("plan", s);
  count_launch();
#define CMM_SEG_LAYOUT(T)                                                                          \
  k_plan_seg_layout<T><<<grid, 256, 0, s>>>(dCodesA, dCodesB, n_a, n_b, logL, logR2, logM, R2,      \
                                            sortedA.as<uint32_t>(), sortedB.as<uint32_t>(),         \
                                            cut.as<uint32_t>(), (int)SA, (int)SB, P.srcA.as<uint32_t>(), \
                                            P.srcB.as<uint32_t>(), P.codeA.as<T>(), P.codeB.as<T>(), \
                                            P.countA.as<uint32_t>(), P.countB.as<uint32_t>())
  if (P.u16) CMM_SEG_LAYOUT(uint16_t);
  else CMM_SEG_LAYOUT(uint32_t);
#undef CMM_SEG_LAYOUT
  CMM_CUDA(cudaGetLastError());
  return P;
}

}  // namespace cmm
