// Internal interface of the batched sketch kernel (cmm_batch.cu), shared by
// the batch plans and the serving engine (cmm_serve.cu).
#pragma once

#include "cmm_internal.h"

namespace cmm {

constexpr int kBatchFftLog = 12;  // largest FFT slab (complex)
constexpr int kBatchWhtLog = 13;  // largest FWHT slab (real, x and y)

// device-side description of one product
struct BProd {
  const void* AT;
  const void* B;
  // per repetition t, the indices of each side stably sorted by slab
  // position h mod L (t-major, SA / SB slots per t): source index | (sign ==
  // +1) << 31, the bucket h itself (u16 when code16), and kPlanThreads + 1
  // cut offsets that split the slots into per-thread runs of whole buckets
  const uint32_t* srcA;
  const uint32_t* srcB;
  const void* codeA;
  const void* codeB;
  const uint32_t* cutA;
  const uint32_t* cutB;
  const int* scale;        // FFT row exponents, n_inner
  const double2* tw;       // w_b^j, j < b
  void* partial;           // [G][d][R][L] (double2 FFT, double FWHT)
  int64_t n_a, n_inner, n_b;
  int SA, SB, code16;
  int d, log2b, logL, logR, G, variant, radix;
  int tc;  // FP32 FWHT: Hadamard-16 stages on the tensor cores (else CUDA cores)
};
// one work item: (product, repetition t, slab r, k-group g)
struct BItem {
  int prod, t, r, g;
};

// one (product, repetition) of the batched k-group reduction + inverse
struct FinJob {
  const void* partial;  // [G][d][R][L] slab partials
  double* p;            // d x b sketch (row t written)
  const double2* tw;    // w_b^j, j < b
  int G, d, t, log2b, logL, variant;
};
// b in [4, 2^14]: the inverse fits one CTA's shared memory
bool batch_finalize_fits(int log2b);
// one launch over n_jobs jobs
void batch_launch_finalize(const FinJob* dJobs, int n_jobs, cudaStream_t s);

// CTAs of the persistent kernel that fit the device at once
int batch_resident_ctas(bool f32);
// one persistent launch over n_items items (counter: one device int, reset here)
void batch_launch_sketch(bool f32, const BProd* dP, const BItem* dI, int n_items, int* dCounter,
                         const double2* tw4096, int ctas, cudaStream_t s);
// the autotuner's cached (slab length, radix) for a product class, if any
bool batch_tuned(int variant, bool f32, int log2b, int64_t n_ab, int* logL, int* radix, int* tc);
// relative cost of one (t, slab, row) unit
double batch_unit_cost(int64_t n_a, int64_t n_b, int logL);

}  // namespace cmm
