/*
 * compmatmul_b200.h -- C ABI of the B200 (sm_100a) compressed matrix
 * multiplication library (libcmm_b200.so).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and
 * returns a cmm_status.  On failure cmm_last_error() gives the message
 * (thread-local).  Status values map one-to-one onto the C++ exceptions of
 * the reference binding: CMM_ERR_INVALID_ARGUMENT <-> std::invalid_argument
 * (ValueError in Python), CMM_ERR_RUNTIME <-> std::runtime_error
 * (RuntimeError), CMM_ERR_NO_MEMORY <-> std::bad_alloc (MemoryError).
 *
 * Conventions of the reference (matmul_fft.hpp:19-24, 149-154): AT is
 * n_inner x n_a row-major, B is n_inner x n_b row-major, C = A^T... i.e.
 * C[i][j] = sum_k AT[k][i] * B[k][j], n_a x n_b row-major.  The sketch p is
 * d x b doubles (matmul_sketch::p, matmul_sketch.hpp:518).
 *
 * Hash kinds follow the strings of compmatmul.cpp:97-104.  Seeds follow
 * matmul_sketch.hpp:15-18 (h1 <- seed, h2 <- seed+1, s1 <- seed+2,
 * s2 <- seed+3).  has_seed == 0 draws the seed from the millisecond clock
 * exactly as rng()() does (rng.hpp:54-56, matmul_fft.hpp:30-32).
 *
 * "host" entry points take host pointers, are synchronous, and allocate
 * device memory internally (stream-ordered pool).  "dev" entry points take
 * device pointers and a cudaStream_t (as void*), enqueue work on that
 * stream and return without synchronising.
 */
#ifndef COMPMATMUL_B200_H
#define COMPMATMUL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CMM_OK = 0,
  CMM_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
  CMM_ERR_RUNTIME = 2,          /* std::runtime_error                    */
  CMM_ERR_NO_MEMORY = 3,        /* std::bad_alloc                        */
  CMM_ERR_CUDA = 4,             /* a CUDA call failed (no reference twin) */
  CMM_ERR_UNSUPPORTED = 5       /* valid for the reference, beyond this build's limits */
} cmm_status;

typedef enum {
  CMM_HASH_MULTIPLY_SHIFT = 0,     /* "multiply shift",     hashing.hpp:27-102  */
  CMM_HASH_MULTIPLY_ADD_SHIFT = 1, /* "multiply add shift", hashing.hpp:111-183 (default) */
  CMM_HASH_TABULATION8 = 2,        /* "tabulation8",        hashing.hpp:232-320 */
  CMM_HASH_TABULATION16 = 3        /* "tabulation16",       hashing.hpp:232-320 */
} cmm_hash_kind;

typedef enum {
  CMM_VARIANT_FFT = 0, /* cyclic convolution, matmul_fft.hpp  */
  CMM_VARIANT_FWHT = 1 /* XOR convolution,     matmul_fwht.hpp */
} cmm_variant;

/* Message of the last failing call on this thread ("" if none). */
const char* cmm_last_error(void);
/* Library version string. */
const char* cmm_version(void);
/* Number of CUDA devices visible (0 if none); never fails. */
int cmm_device_count(void);

/* Largest b the sketch kernels accept (2^24); larger powers of two give
 * CMM_ERR_UNSUPPORTED. */
int cmm_max_buckets(void);

/* ---------------------------------------------------------------------
 * Host-pointer drop-ins of the reference's header entry points.
 * ------------------------------------------------------------------- */

/* Replaces compmatmul::matmul_fft<H> (matmul_fft.hpp:155-178) and
 * compmatmul::matmul_fwht<H> (matmul_fwht.hpp:144-167): compressed product
 * followed by dense median decompression into C (n_a x n_b).  Argument
 * checks of compmatmul.cpp:87-105 (b power of two > 1, d >= 1, hash). */
int cmm_matmul(int variant, int hash_kind, int64_t n_a, int64_t n_inner, int64_t n_b, double* C,
               const double* AT, const double* B, int d, int b, int has_seed, uint64_t seed);

/* Replaces compmatmul::matmul_compressed_product_fft<H> (matmul_fft.hpp:25-129)
 * and _fwht<H> (matmul_fwht.hpp:25-114): writes the d x b sketch p to p_out
 * (host) and the seed actually used to *seed_out (may be NULL). */
int cmm_compressed_product(int variant, int hash_kind, int64_t n_a, int64_t n_inner, int64_t n_b,
                           const double* AT, const double* B, int d, int b, int has_seed,
                           uint64_t seed, double* p_out, uint64_t* seed_out);

/* Replaces compmatmul::matmul_decompress_fft<H> / _fwht<H>
 * (matmul_fft.hpp:135-147, matmul_fwht.hpp:122-134) for `count` entries
 * (i[e], j[e]): out[e] = median_t s1_t(i) s2_t(j) p_t[idx], idx = (h1+h2)&(b-1)
 * (FFT) or h1^h2 (FWHT).  p is the host d x b sketch drawn with `seed`. */
int cmm_decompress(int variant, int hash_kind, int d, int b, uint64_t seed, const double* p,
                   int64_t count, const uint32_t* i, const uint32_t* j, double* out);

/* Replaces compmatmul::array::matmul_gemm<double> (array.hpp:85-95) behind
 * the Python `gemm` (compmatmul.cpp:76-85): exact C = AT^T B in FP64. */
int cmm_gemm(int64_t n_a, int64_t n_inner, int64_t n_b, double* C, const double* AT,
             const double* B);

/* Bucket/sign codes of one side of the sketch for keys 0..n-1 (host
 * output, d x n): code = bucket | (sign == +1) << 31; side 0 = (h1,s1),
 * side 1 = (h2,s2).  Exposes hashing.hpp operator()/sign as computed on the
 * GPU (the same codes the sketch kernels use). */
int cmm_hash_codes(int hash_kind, int d, int b, uint64_t seed, int side, int64_t n,
                   uint32_t* codes_out);

/* ---------------------------------------------------------------------
 * Host-side random stream and hash draws (no CUDA call).  They let the C++
 * header entry points hand out the reference's rng and hash objects
 * (matmul_sketch::h1/h2/s1/s2) with the same parameters bit for bit.
 * ------------------------------------------------------------------- */

/* Replaces compmatmul::splitmix64 + rng::rng(seed) (rng.hpp:26-33, 54-57):
 * the four xoshiro256** state words seeded from `seed`. */
void cmm_rng_seed(uint64_t seed, uint64_t* state4);
/* Replaces rng::operator() (rng.hpp:59-72): the next 64-bit value; steps
 * the state in place. */
uint64_t cmm_rng_next(uint64_t* state4);
/* Replaces compmatmul::current_system_time_millis (rng.hpp:40-44), the
 * seed of rng() without one. */
uint64_t cmm_time_millis(void);
/* Replaces Hash::draw(n, buckets, seed) of hashing.hpp (multiply_shift
 * :69-87, multiply_add_shift :145-160, tabulation :277-295): parameters of
 * n functions from one stream seeded with `seed`, packed back to back:
 * multiply shift -> u64 a; multiply add shift -> u64 a, u64 b;
 * tabulation8 -> u32 T[4][256]; tabulation16 -> u32 T[2][65536].
 * buckets must be a power of two (the reference's message otherwise). */
int cmm_hash_params(int hash_kind, int n, uint64_t buckets, uint64_t seed, void* out,
                    size_t out_bytes);

/* ---------------------------------------------------------------------
 * Device-pointer, stream-ordered entry points (no reference twin: the
 * reference is host-only).  All pointers are device pointers.
 * ------------------------------------------------------------------- */

/* Sketch only: dP (d x b FP64) from dAT, dB. */
int cmm_dev_compressed_product(int variant, int hash_kind, int64_t n_a, int64_t n_inner,
                               int64_t n_b, const double* dAT, const double* dB, int d, int b,
                               uint64_t seed, double* dP, void* stream);

/* Allocation-free twin of cmm_dev_compressed_product; it has no counterpart
 * in the reference (which allocates its sketches on the host heap,
 * matmul_fft.hpp / matmul_fwht.hpp).  For callers that cannot call
 * cudaMalloc: a plugin whose host framework owns all device memory and
 * forbids allocation after set-up, or a serving loop whose pool already
 * holds the HBM (cudaMalloc would fail or break its budget, and cudaFree
 * synchronises the whole device, stalling every other stream).
 *   - It calls no cudaMalloc / cudaMallocAsync / cudaFree and no allocating
 *     library routine: every intermediate (hash parameters, codes, row
 *     scales, twiddles, k-group partials, inverse work) lives in one
 *     file-scope device array of CMM_NOALLOC_SCRATCH_BYTES per device.
 *     The host side draws the hash parameters and twiddles into ordinary
 *     host memory and copies them in with cudaMemcpyAsync.
 *   - Scratch needed, in bytes (each term rounded up to 256):
 *       4 * d * param_bytes(hash) + 4 * d * n_a + 4 * d * n_b
 *       + 4 * n_inner (FFT only) + 16 * b + 2 * d * b * e + d * b * e,
 *     e = 16 (FFT) or 8 (FWHT); param_bytes = 8 (MS), 16 (MAS), 4096
 *     (tab8), 524288 (tab16).  Larger products return CMM_ERR_UNSUPPORTED
 *     before any CUDA call, with the bytes needed in cmm_last_error().
 *   - The first call on a device looks up the scratch address
 *     (cudaGetSymbolAddress, once per device); make that first call before
 *     any stream capture begins.
 *   - The k-group partials are cleared on every call; all other scratch is
 *     fully written before it is read.
 *   - Calls that overlap in time on one device (other streams, other host
 *     threads) race on the one scratch array: serialise them. */
#define CMM_NOALLOC_SCRATCH_BYTES (32u << 20)
int cmm_dev_compressed_product_noalloc(int variant, int hash_kind, int64_t n_a, int64_t n_inner,
                                       int64_t n_b, const double* dAT, const double* dB, int d,
                                       int b, uint64_t seed, double* dP, void* stream);

/* Device-resident sketch queries (matmul_decompress_fft/fwht on a device
 * sketch, matmul_fft.hpp:135-147 / matmul_fwht.hpp:122-134): the median
 * estimate of `count` listed entries (dI[e], dJ[e]) into dOut. */
int cmm_dev_decompress_entries(int variant, int hash_kind, int d, int b, uint64_t seed, const double* dP,
                               int64_t count, const uint32_t* dI, const uint32_t* dJ, double* dOut,
                               void* stream);
/* Top-K entries of the n_a x n_b median estimate of sketch dP without the
 * dense matrix: rows are decompressed in tiles of at most scratch_bytes
 * (0: 256 MiB; at least K entries), each tile's top-K is kept and the lists
 * are merged.  Same result and order as cmm_dev_topk on the dense estimate
 * (value descending, ties by (i, j) ascending).  K <= 4096; synchronises. */
int cmm_dev_sketch_topk(int variant, int hash_kind, int64_t n_a, int64_t n_b, int d, int b, uint64_t seed,
                        const double* dP, int K, size_t scratch_bytes, uint32_t* d_i, uint32_t* d_j, double* d_v,
                        void* stream);

/* Dense median decompression of dP into dC (n_a x n_b FP64). */
int cmm_dev_decompress_dense(int variant, int hash_kind, int64_t n_a, int64_t n_b, int d, int b,
                             uint64_t seed, const double* dP, double* dC, void* stream);

/* Compressed product + dense decompression (matmul_fft / matmul_fwht). */
int cmm_dev_matmul(int variant, int hash_kind, int64_t n_a, int64_t n_inner, int64_t n_b,
                   double* dC, const double* dAT, const double* dB, int d, int b, uint64_t seed,
                   void* stream);

/* Top-K entries of a dense n_a x n_b FP64 matrix on the device, by value
 * descending, ties by (i, j) ascending.  Writes K (i, j, value) triples to
 * device arrays.  Synchronises `stream` (the candidate count is read back). */
int cmm_dev_topk(const double* dC, int64_t n_a, int64_t n_b, int K, uint32_t* d_i, uint32_t* d_j,
                 double* d_v, void* stream);

/* Exact FP64 C = AT^T B on the device. */
int cmm_dev_gemm(int64_t n_a, int64_t n_inner, int64_t n_b, double* dC, const double* dAT,
                 const double* dB, void* stream);

/* ---------------------------------------------------------------------
 * Mixed precision (no reference twin: the reference binding accepts FP64
 * only, compmatmul.cpp:22-30).  FP32 inputs; sketches and transforms in
 * FP32 with two-sum compensated accumulation over k; FWHT Hadamard-16
 * factors on the tensor cores (BF16 hi/lo split, FP32 accumulation); the
 * reduction of the d spectra, the inverse transform, p and C in FP64.
 * ------------------------------------------------------------------- */
int cmm_dev_compressed_product_f32(int variant, int hash_kind, int64_t n_a, int64_t n_inner,
                                   int64_t n_b, const float* dAT, const float* dB, int d, int b,
                                   uint64_t seed, double* dP, void* stream);
int cmm_dev_matmul_f32(int variant, int hash_kind, int64_t n_a, int64_t n_inner, int64_t n_b,
                       double* dC, const float* dAT, const float* dB, int d, int b, uint64_t seed,
                       void* stream);
int cmm_compressed_product_f32(int variant, int hash_kind, int64_t n_a, int64_t n_inner,
                               int64_t n_b, const float* AT, const float* B, int d, int b,
                               int has_seed, uint64_t seed, double* p_out, uint64_t* seed_out);
int cmm_matmul_f32(int variant, int hash_kind, int64_t n_a, int64_t n_inner, int64_t n_b,
                   double* C, const float* AT, const float* B, int d, int b, int has_seed,
                   uint64_t seed);
/* Batched forward Walsh-Hadamard transform of FP32 rows on device memory:
 * y[r] = H x[r] for r < rows, each row 2^log2n floats (log2n 11..13), H
 * the unnormalised natural-order (Sylvester) matrix.  Replaces
 * fwht_transformer::forward (transform.hpp:94-144, FXT walsh_wak in natural
 * order; golden values tests.cpp:621-671) for FP32 rows.  method 0: every
 * stage on CUDA cores; method 1: the two Hadamard-16 stages as tcgen05.mma
 * on BF16 hi/mid/lo splits with FP32 accumulators in tensor memory, the
 * rest on CUDA cores.  x == y is allowed; x and y 16-byte aligned.
 * Synchronous on `stream`: returns once y is written, so that a tensor-core
 * completion wait that ran out (CMM_ERR_RUNTIME) is reported. */
int cmm_dev_wht_rows_f32(const float* x, float* y, int64_t rows, int log2n, int method,
                         void* stream);

/* ---------------------------------------------------------------------
 * Batched products (no reference twin: the reference computes one product
 * per call).  A batch plan fixes a list of independent products of uneven
 * shape -- each with its own variant, hash family, d, b, seed, sizes and
 * device buffers -- and runs all of them per cmm_batch_run:
 *   hash codes of every product (one launch), per-k row balance of the FFT
 *   products (one launch), ONE persistent sketch launch whose CTAs pop work
 *   items (product, repetition t, frequency slab, k-group) from a device
 *   queue ordered longest first, then each product's k-group reduction +
 *   inverse and (when C != NULL) dense median decompression.
 * The whole sequence is captured in a CUDA graph on the first run and
 * replayed afterwards.  Per product class (variant, precision, b, sizes) an
 * autotuner times the candidate slab lengths and transform radices on the
 * product's own data and caches the fastest (process-wide); the number of
 * k-groups, hence CTAs per product, follows from the tuned per-row costs.
 * Each product must have b <= 2^24; the device buffers must stay valid and
 * unchanged in address for the plan's lifetime (their contents may change
 * between runs).  Results equal cmm_dev_compressed_product /
 * cmm_dev_matmul (FP64) or their _f32 forms on the same inputs, within
 * the tolerances those state.
 * ------------------------------------------------------------------- */
typedef struct {
  int variant;      /* CMM_VARIANT_FFT or CMM_VARIANT_FWHT */
  int hash_kind;    /* cmm_hash_kind */
  int d, b;
  int64_t n_a, n_inner, n_b;
  uint64_t seed;
  const void* AT;   /* device, n_inner x n_a; float64, or float32 when the plan is f32 */
  const void* B;    /* device, n_inner x n_b; same type */
  double* p;        /* device, d x b sketch (output) */
  double* C;        /* device, n_a x n_b dense estimate (output), or NULL for the sketch only */
} cmm_batch_product;

/* tune != 0 runs the autotuner for product classes not yet in its cache. */
int cmm_batch_create(const cmm_batch_product* products, int count, int f32, int tune,
                     void** handle);
/* Runs every product of the plan on `stream` (NULL: an internal stream,
 * synchronised before returning). */
int cmm_batch_run(void* handle, void* stream);
/* Work items of the persistent launch, its CTAs, and the kernel launches
 * (graph kernel nodes) per run. */
int cmm_batch_info(void* handle, int64_t* items, int* ctas, int* launches);
/* The configuration chosen for one product: log2 of the slab length, the
 * transform radix (4 or 8), the k-groups, and whether the autotuner timed it. */
int cmm_batch_config(void* handle, int product, int* log2_slab, int* radix, int* groups,
                     int* tuned);
int cmm_batch_destroy(void* handle);

/* ---------------------------------------------------------------------
 * Serving (no reference twin): continuous batching of independent
 * compressed products.  A background scheduler admits submitted requests in
 * arrival order while the device memory they hold stays under the cap
 * (inputs when copied in, hash codes, sorted plans, row balance, k-group
 * partials, the sketch), prepares each on an upload stream, groups the
 * prepared ones into waves -- each wave is one persistent sketch launch over
 * all of its products' work items plus their reduction + inverse -- and runs
 * waves on several streams at once, so requests that arrive while others
 * run are admitted as memory frees up and their work overlaps on the device.
 * The sketch p of each request is copied back to the caller's host buffer.
 * A request's result does not depend on what it was batched with: its work
 * items and their order are fixed by the request alone.
 * ------------------------------------------------------------------- */
typedef struct {
  size_t mem_cap_bytes;  /* admission cap on device bytes held by admitted requests */
  int f32;               /* 1: float32 inputs (mixed precision); 0: float64 */
  int streams;           /* waves in flight at once (>= 1) */
  int max_wave;          /* most requests per wave (>= 1) */
  size_t cache_bytes;    /* device bytes for hash codes + sorted plans kept across requests
                            with the same (hash, seed, d, b, n_a, n_b); 0 disables the cache */
} cmm_server_config;

typedef struct {
  int variant, hash_kind, d, b;
  int64_t n_a, n_inner, n_b;
  uint64_t seed;
  const void* AT;      /* n_inner x n_a, float32 or float64 per the server */
  const void* B;       /* n_inner x n_b */
  int inputs_on_device; /* 1: AT, B are device pointers; 0: host (pinned host memory copies asynchronously) */
  double* p;           /* host d x b output */
} cmm_request;

typedef struct {
  int64_t submitted, completed, queued, in_flight;
  int64_t waves, max_waves_in_flight;
  size_t mem_in_use, max_mem_in_use;
  int64_t cache_hits, cache_misses;
  size_t cache_in_use;
} cmm_server_stats;

int cmm_server_create(const cmm_server_config* cfg, void** server);
/* Queues one request (its buffers must stay valid until it completes);
 * *id identifies it.  A request that alone needs more than the cap is
 * rejected with CMM_ERR_INVALID_ARGUMENT. */
int cmm_server_submit(void* server, const cmm_request* req, uint64_t* id);
/* Waits up to timeout_s seconds (< 0: no limit) for request id; *done = 1
 * when its p is in the host buffer.  *latency_s (may be NULL) = submit to
 * completion, seconds. */
int cmm_server_wait(void* server, uint64_t id, double timeout_s, int* done, double* latency_s);
int cmm_server_stats_get(void* server, cmm_server_stats* out);
/* Drains every queued request, then stops the scheduler and frees all. */
int cmm_server_destroy(void* server);

/* ---------------------------------------------------------------------
 * Instrumentation for benchmarks (no reference twin).  When enabled, every
 * kernel launch of a family is bracketed by CUDA events recorded on the
 * stream it is launched on.  Families: "hash", "scale", "plan",
 * "materialize", "sketch", "finalize", "decompress", "topk", "gemm".
 * ------------------------------------------------------------------- */
void cmm_profile_enable(int on);
void cmm_profile_reset(void);
/* Sum of event-timed milliseconds and number of timed launches of a family
 * since the last reset; waits for the recorded events. */
int cmm_profile_read(const char* family, double* total_ms, int64_t* launches);
/* Kernels launched by this library since load (always counted). */
int64_t cmm_launch_count(void);
/* Name of the sketch kernel family the last compressed product on this host
 * thread ran ("cluster", "slab", "slab-mixed", "small-b"); "" before any. */
const char* cmm_last_sketch_kernel(void);
/* Measured FMA throughput of the current device in TFLOP/s (2 flops per
 * FMA; FP64 if fp64 != 0, else FP32), from a register-resident FMA loop
 * timed with CUDA events: the arithmetic roofline's denominator. */
int cmm_probe_fma_tflops(int fp64, double* tflops);
/* Per-phase cycles of the cluster sketch kernel, summed over its CTAs and
 * inner indices since the last call (then cleared): cycles[0..5] = clearing
 * the sub-spectrum buffer, waiting for the staged row, the scatter, the
 * local radix passes, the cluster barrier, the combine + accumulation;
 * *steps = (CTA, inner index) pairs timed.  Only in a library built with
 * -DCMM_PHASE_CLOCKS (CMM_EXTRA_NVFLAGS); otherwise CMM_ERR_UNSUPPORTED. */
int cmm_cluster_phase_cycles(double* cycles, double* steps);

#ifdef __cplusplus
}
#endif

#endif /* COMPMATMUL_B200_H */
