// Internal declarations shared by the host runtime (cmm_capi.cu) and the
// kernel translation units.  Not part of the public ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/compmatmul_b200.h"

namespace cmm {

// ------------------------------------------------------------------ errors
// Exceptions thrown inside the runtime; the C ABI turns them into status
// codes (compmatmul_b200.h).
struct invalid_argument : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};
struct runtime_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct unsupported : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct cuda_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void cuda_check(cudaError_t e, const char* what);
#define CMM_CUDA(call) ::cmm::cuda_check((call), #call)

// ------------------------------------------------------- rng and hashing
// xoshiro256** seeded by splitmix64 (rng.hpp:26-33, 59-72).
struct Xoshiro256ss {
  uint64_t s[4];
  explicit Xoshiro256ss(uint64_t seed);
  uint64_t operator()();
};

// Milliseconds since the epoch (rng.hpp:40-44).
uint64_t time_millis();
// Seed used when the caller gives none: rng()() with the ms clock seed
// (rng.hpp:40-44, 54-56; matmul_fft.hpp:30-32).
uint64_t time_seed();

enum HashKind { MS = 0, MAS = 1, TAB8 = 2, TAB16 = 3 };

size_t hash_param_bytes(int kind);

// Parameters of `n` functions of family `kind` drawn from one stream
// seeded with `seed` (hashing.hpp:69-87, 145-160, 277-295), packed as the
// device kernels read them: MS -> n x u64 a; MAS -> n x (u64 a, u64 b);
// TAB8 -> n x u32[4][256]; TAB16 -> n x u32[2][65536].
std::vector<uint8_t> draw_hash_params(int kind, int n, uint64_t seed);

// The four function sets of one sketch (matmul_sketch.hpp:15-18), each d
// functions: order h1, h2, s1, s2.  One contiguous host blob.
struct SketchParams {
  int kind = 0, d = 0, b = 0, log2b = 0;
  uint64_t seed = 0;
  size_t fn_bytes = 0;  // bytes per function
  std::vector<uint8_t> blob;  // [h1 | h2 | s1 | s2], each d * fn_bytes
};
SketchParams make_sketch_params(int kind, int d, int b, uint64_t seed);

// ------------------------------------------------------ host copies
// Copies between device memory and caller-owned host memory (cmm_hostcopy.cpp).
// Pinned host memory: cudaMemcpyAsync on cs.  Pageable host memory: through
// pinned staging slots filled / drained by several host threads;
// host_to_device returns once the source has been read, device_to_host once
// dst holds the data (pinned: enqueued only).
void host_to_device(void* dst, const void* src, size_t bytes, cudaStream_t cs);
void device_to_host(void* dst, const void* src, size_t bytes, cudaStream_t cs);

// ---------------------------------------------------------- device pool
// Stream-ordered scratch allocation (cudaMallocAsync) with RAII release.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  DevBuf() = default;
  DevBuf(size_t n, cudaStream_t s);
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept;
  ~DevBuf();
  template <typename T>
  T* as() const { return static_cast<T*>(ptr); }
};

// --------------------------------------------------------- kernel plans
constexpr int kVariantFFT = 0;
constexpr int kVariantFWHT = 1;

// Largest sub-transform length held in one CTA's shared memory.
constexpr int kFftLmaxLog = 12;   // 4096 complex FP64 (64 KB) + accumulator
constexpr int kFwhtLmaxLog = 13;  // 8192 real FP64 x 2 (128 KB) + accumulator
constexpr int kMaxLog2B = 24;     // b <= 2^24 (R = b/L <= 4096)

// Static scratch of the allocation-free entry point (32 MiB per device).
constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;
void* noalloc_scratch();  // its device address, looked up once per device

struct SketchPlan {
  int variant, d, b, log2b;
  int logL, L;       // sub-transform length L = b / R
  int logR, R;       // number of frequency slabs (CTAs) per repetition
  int KB;            // sequences per CTA pass (KB * L = capacity)
  int G;             // number of k groups
  int64_t n_a, n_inner, n_b;
};
SketchPlan plan_sketch(int variant, int64_t n_a, int64_t n_inner, int64_t n_b, int d, int b,
                       int num_sms);

// Device-resident per-b twiddle table w[j] = exp(-2 pi i j / b), j < b
// (double2), built on the host in long double and cached per (device, b).
const double2* twiddles(int b, cudaStream_t s);

// ------------------------------------------------------------- launchers
void launch_hash_codes(int kind, const void* dHfns, const void* dSfns, int d, int log2b,
                       int64_t n, uint32_t* dCodes, cudaStream_t s);
// codes of explicit keys (dKeys[e]) instead of 0..n-1
void launch_hash_codes_keys(int kind, const void* dHfns, const void* dSfns, int d, int log2b,
                            int64_t n, const uint32_t* dKeys, uint32_t* dCodes, cudaStream_t s);

// one code set of a batch: codes (d x n) of keys 0..n-1 under (H, S)
struct HashJob {
  const void* H;
  const void* S;
  uint32_t* codes;
  int64_t n;
  int d, log2b, kind;
};
void launch_hash_codes_jobs(const HashJob* dJobs, int njobs, int64_t max_total, cudaStream_t s);

void launch_row_scale(const double* dAT, const double* dB, int64_t n_a, int64_t n_inner,
                      int64_t n_b, int* dScaleExp, cudaStream_t s);

void launch_sketch_accumulate(const SketchPlan& P, const double* dAT, const double* dB,
                              const uint32_t* dCodesA, const uint32_t* dCodesB,
                              const int* dScaleExp, const double2* dTw, void* dPartial,
                              cudaStream_t s);

void launch_finalize(const SketchPlan& P, const void* dPartial, const double2* dTw,
                     void* dWork, double* dP, cudaStream_t s);

void launch_decompress_dense(int variant, int d, int b, int64_t n_a, int64_t n_b,
                             const uint32_t* dCodesA, const uint32_t* dCodesB, const double* dP,
                             double* dC, cudaStream_t s);
void launch_decompress_dense_rows(int variant, int d, int b, int64_t n_a, int64_t n_b, int64_t i0,
                                  int64_t rows, const uint32_t* dCodesA, const uint32_t* dCodesB,
                                  const double* dP, double* dCrows, cudaStream_t s);

// codes are d x count, one column per listed (i, j) entry
void launch_decompress_list(int variant, int d, int b, int64_t count, const uint32_t* dCodesI,
                            const uint32_t* dCodesJ, const double* dP, double* dOut,
                            cudaStream_t s);

void launch_gemm(int64_t n_a, int64_t n_inner, int64_t n_b, double* dC, const double* dAT,
                 const double* dB, cudaStream_t s);

// ---------------------------------------------------------- slab plans
// Bucket-sorted, thread-interleaved slot layout of one sketch (see
// cmm_plan.cu) and its per-t materialized rows (sketch kernels v1).
constexpr int kPlanThreads = 512;          // threads of the v1 sketch kernels
constexpr uint32_t kPadSlot = 0xffffffffu;  // slot without an index
struct SlabPlan {
  int d = 0, logL = 0, EA = 0, EB = 0;
  int segs = 1;     // residue segments per (t, side): R2 for the cluster kernels
  bool compact = false;  // residue plans: segments in sorted order, EA/EB = slots per segment,
                         // countA/countB hold kPlanThreads + 1 cut offsets per segment
  // slots of one materialized row per t and side
  int64_t slots_a() const { return (int64_t)segs * EA * (compact ? 1 : kPlanThreads); }
  int64_t slots_b() const { return (int64_t)segs * EB * (compact ? 1 : kPlanThreads); }
  bool u16 = true;  // codes stored as u16 (b <= 2^16)
  int64_t n_a = 0, n_b = 0;
  DevBuf srcA, srcB;      // d x S: index | (sign == +1) << 31, or kPadSlot
  DevBuf codeA, codeB;    // d x S: bucket h
  DevBuf countA, countB;  // d x kPlanThreads: slots used per thread
};
SlabPlan make_slab_plan(const uint32_t* dCodesA, const uint32_t* dCodesB, int64_t n_a, int64_t n_b,
                        int d, int b, int logL, cudaStream_t s);
// residue plans for the cluster kernels (b = R1 * R2 * L)
SlabPlan make_residue_plan(const uint32_t* dCodesA, const uint32_t* dCodesB, int64_t n_a, int64_t n_b,
                           int d, int b, int logL, int logR2, cudaStream_t s);
void launch_materialize(const SlabPlan& P, const double* dAT, const double* dB, int64_t k0,
                        int64_t kc, double* dOutA, double* dOutB, cudaStream_t s);
// v1 sketch over materialized rows of inner indices [k0, k0 + kc) (chunk);
// accumulate != 0 adds to the partials instead of overwriting them.
void launch_sketch_v1(const SketchPlan& SP, const SlabPlan& P, const double* dMatA,
                      const double* dMatB, int64_t kc, const int* dScaleExp, int64_t k0,
                      const double2* dTw, void* dPartial, int accumulate, cudaStream_t s);
SketchPlan plan_sketch_v1(int variant, int64_t n_a, int64_t n_inner, int64_t n_b, int d, int b,
                          int sms);
// true if the v1 kernels handle this (variant, b, n) and sizes
bool sketch_v1_applicable(int variant, int b, int64_t n_a, int64_t n_b);

// Mixed precision (FP32 inputs, FP32 transforms, compensated accumulation,
// FP64 reduction and inverse): slabs of L = 8192 (cmm_sketch_mixed.cu).
SketchPlan plan_sketch_mixed(int variant, int64_t n_a, int64_t n_inner, int64_t n_b, int d, int b,
                             int sms);
bool sketch_mixed_applicable(int variant, int b);
void launch_sketch_mixed(const SketchPlan& SP, const SlabPlan& P, const float* dMatA,
                         const float* dMatB, int64_t kc, const int* dScaleExp, int64_t k0,
                         const double2* dTw, void* dPartial, int accumulate, cudaStream_t s);
void launch_row_scale_f32(const float* dAT, const float* dB, int64_t n_a, int64_t n_inner,
                          int64_t n_b, int* dScaleExp, cudaStream_t s);
void launch_materialize_f32(const SlabPlan& P, const float* dAT, const float* dB, int64_t k0,
                            int64_t kc, float* dOutA, float* dOutB, cudaStream_t s);
void launch_f32_to_f64(const float* src, double* dst, int64_t n, cudaStream_t s);

// Cluster kernels (cmm_sketch_cluster.cu): b = R1 * R2 * L; partials in
// natural frequency order [g][t][b].
struct ClusterPlan {
  int logL = 0, log2b = 0, logR1 = 0, logR2 = 0, G = 1, max_clusters = 0;
  int nt = 512;  // threads per CTA: 512, or 256 (FP64, two CTAs per SM)
};
bool sketch_cluster_applicable(int variant, bool f32, int b);
ClusterPlan plan_cluster(int variant, bool f32, int64_t n_inner, int d, int b, int64_t n_a, int64_t n_b);
bool cluster_smem_fits(int variant, bool f32, const ClusterPlan& C, const SlabPlan& P);
void launch_sketch_cluster(int variant, bool f32, const ClusterPlan& C, const SlabPlan& P,
                           const void* dMatA, const void* dMatB, int64_t kc, const int* dScaleExp,
                           int64_t k0, const double2* dTw, void* dPartial, int d, int accumulate,
                           cudaStream_t s);
// true (and cleared) when a group barrier wait of a cluster-kernel launch
// ran out since the last call; that launch wrote NaN partials
bool sketch_group_timed_out();
// per-phase cycle sums of the cluster kernel (CMM_PHASE_CLOCKS builds only)
bool cluster_phase_cycles(double* cycles6, double* steps);
// finalize for partials in natural frequency order (cluster kernels)
void launch_finalize_natural(int variant, int d, int b, int G, const void* dPartial,
                             const double2* dTw, void* dWork, double* dP, cudaStream_t s);

// Batched products (cmm_batch.cu); the product descriptor is the public
// cmm_batch_product of compmatmul_b200.h.
struct BatchPlan;
BatchPlan* batch_create(const cmm_batch_product* products, int count, bool f32, bool tune);
void batch_run(BatchPlan* B, cudaStream_t stream);
void batch_info(const BatchPlan* B, int64_t* items, int* ctas, int* launches);
void batch_config(const BatchPlan* B, int i, int* log2_slab, int* radix, int* groups, int* tuned);
void batch_destroy(BatchPlan* B);

// Serving engine (cmm_serve.cu)
struct Server;
Server* server_create(const cmm_server_config* cfg);
uint64_t server_submit(Server* S, const cmm_request* req);
bool server_wait(Server* S, uint64_t id, double timeout_s, double* latency_s);
void server_stats(Server* S, cmm_server_stats* out);
void server_destroy(Server* S);

// Top-K over a dense matrix; returns after synchronising s.
void topk_dense(const double* dC, int64_t n_a, int64_t n_b, int K, uint32_t* dI, uint32_t* dJ,
                double* dV, cudaStream_t s);

int num_sms();

// ------------------------------------------------------- instrumentation
// Event timing of kernel families (cmm_profile_*) and the launch counter.
void prof_begin(const char* family, cudaStream_t s);
void prof_end(const char* family, cudaStream_t s);
void count_launch(int n = 1);
void set_sketch_kernel(const char* name);  // recorded for cmm_last_sketch_kernel
bool prof_set(bool on);                    // event profiling on/off; returns the previous state
double probe_fma_tflops(bool fp64, cudaStream_t s);
// batched FP32 natural-order WHT of rows of 2^log2n (cmm_wht_tc.cu); synchronous on s
void wht_rows_f32(const float* x, float* y, int64_t rows, int log2n, int method, cudaStream_t s);
struct ProfScope {
  const char* fam;
  cudaStream_t s;
  ProfScope(const char* f, cudaStream_t st) : fam(f), s(st) { prof_begin(fam, s); }
  ~ProfScope() { prof_end(fam, s); }
};

}  // namespace cmm
