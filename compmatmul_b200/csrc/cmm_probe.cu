// Measured FMA peak of this device (the denominator of the arithmetic
// roofline of the sketch kernels): every thread runs kChains independent
// FMA chains for `iters` steps; 2 flops per FMA; timed with CUDA events
// around the second of two launches.
#include "cmm_internal.h"

namespace cmm {
namespace {

constexpr int kChains = 8;
constexpr int kProbeThreads = 512;

template <typename T>
__global__ void __launch_bounds__(kProbeThreads) k_fma_probe(int iters, T* sink) {
  T x[kChains];
  const T a = (T)0.999999, c = (T)1e-7;
#pragma unroll
  for (int e = 0; e < kChains; ++e) x[e] = (T)(threadIdx.x + e) * (T)1e-3;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int e = 0; e < kChains; ++e) x[e] = fma(x[e], a, c);
  }
  T s = 0;
#pragma unroll
  for (int e = 0; e < kChains; ++e) s += x[e];
  if (s == (T)-1) sink[0] = s;  // never true; keeps the chains live
}

template <typename T>
double probe(cudaStream_t s) {
  const int sms = num_sms();
  const int blocks = sms * 4, iters = 1 << 14;
  DevBuf sink(sizeof(T), s);
  cudaEvent_t e0, e1;
  CMM_CUDA(cudaEventCreate(&e0));
  CMM_CUDA(cudaEventCreate(&e1));
  float ms = 0.f;
  for (int rep = 0; rep < 2; ++rep) {
    CMM_CUDA(cudaEventRecord(e0, s));
    k_fma_probe<T><<<blocks, kProbeThreads, 0, s>>>(iters, sink.as<T>());
    CMM_CUDA(cudaGetLastError());
    CMM_CUDA(cudaEventRecord(e1, s));
    CMM_CUDA(cudaEventSynchronize(e1));
    CMM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double flops = 2.0 * kChains * (double)iters * (double)blocks * kProbeThreads;
  return flops / (ms * 1e-3) / 1e12;
}

}  // namespace

double probe_fma_tflops(bool fp64, cudaStream_t s) { return fp64 ? probe<double>(s) : probe<float>(s); }

}  // namespace cmm
