// Host runtime and C ABI of libcmm_b200.so (declared in
// include/compmatmul_b200.h).  Validates arguments with the reference's
// rules and messages (compmatmul.cpp:87-105), draws hash parameters on the
// host (bit-exact with hashing.hpp), and runs the device pipeline:
//   hash codes -> row balance (FFT) -> fused sketch/transform/accumulate
//   -> k-group reduction + inverse -> (median decompression) -> (top-K).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>

#include "../../include/compmatmul_b200.h"
#include "cmm_internal.h"

namespace cmm {

static thread_local std::string g_last_error;

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    if (e == cudaErrorMemoryAllocation) throw std::bad_alloc();
    throw cuda_error(std::string("CUDA error: ") + cudaGetErrorString(e) + " in " + what);
  }
}

static void configure_pool();

DevBuf::DevBuf(size_t n, cudaStream_t s) : bytes(n), stream(s) {
  if (n) {
    configure_pool();
    CMM_CUDA(cudaMallocAsync(&ptr, n, s));
  }
}
DevBuf& DevBuf::operator=(DevBuf&& o) noexcept {
  if (this != &o) {
    if (ptr) cudaFreeAsync(ptr, stream);
    ptr = o.ptr; bytes = o.bytes; stream = o.stream;
    o.ptr = nullptr; o.bytes = 0;
  }
  return *this;
}
DevBuf::~DevBuf() {
  if (ptr) cudaFreeAsync(ptr, stream);
}

int num_sms() {
  static std::mutex mu;
  static std::map<int, int> cache;
  int dev = 0;
  CMM_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  int n = 0;
  CMM_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  cache[dev] = n;
  return n;
}

// w[j] = exp(-2 pi i j / b), j < b, built in long double once per b on the
// host (kept for the process: the device tables and the allocation-free
// entry point copy from it)
static const std::vector<double2>& host_twiddles(int b) {
  static std::mutex mu;
  static std::map<int, std::vector<double2>> cache;
  std::lock_guard<std::mutex> g(mu);
  auto it = cache.find(b);
  if (it != cache.end()) return it->second;
  std::vector<double2> h((size_t)b);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int j = 0; j < b; ++j) {
    const long double a = -two_pi * (long double)j / (long double)b;
    h[(size_t)j] = make_double2((double)cosl(a), (double)sinl(a));
  }
  return cache.emplace(b, std::move(h)).first->second;
}

// the same table on the device, cached per (device, b)
const double2* twiddles(int b, cudaStream_t s) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, double2*> cache;
  int dev = 0;
  CMM_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_pair(dev, b);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  const std::vector<double2>& h = host_twiddles(b);
  double2* d = nullptr;
  CMM_CUDA(cudaMalloc(&d, sizeof(double2) * (size_t)b));
  CMM_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(double2) * (size_t)b, cudaMemcpyHostToDevice, s));
  CMM_CUDA(cudaStreamSynchronize(s));
  cache[key] = d;
  return d;
}

// Keep freed blocks of the device's default stream-ordered pool cached
// (release threshold = max) so repeated calls do not re-map GBs of device
// memory at every synchronisation.  Once per device.
static void configure_pool() {
  static std::mutex mu;
  static std::map<int, bool> done;
  int dev = 0;
  CMM_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  if (done[dev]) return;
  cudaMemPool_t pool;
  CMM_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t thr = ~0ULL;
  CMM_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  done[dev] = true;
}

// one non-blocking stream per (host thread, device) for the host-pointer API
static cudaStream_t host_stream() {
  static thread_local std::map<int, cudaStream_t> streams;
  int dev = 0;
  CMM_CUDA(cudaGetDevice(&dev));
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t s;
  CMM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  streams[dev] = s;
  return s;
}

// --------------------------------------------------------------- checks
static int ilog2_int(int b) {
  int l = 0;
  while ((1 << l) < b) ++l;
  return l;
}

// compmatmul.cpp:87-105 (b, d, hash) plus this build's own limits
static void check_params(int variant, int kind, int d, int b) {
  if (variant != kVariantFFT && variant != kVariantFWHT)
    throw invalid_argument("variant must be CMM_VARIANT_FFT or CMM_VARIANT_FWHT");
  if (b < 2 || (b & (b - 1)) != 0)
    throw invalid_argument("b must be power of 2 greater than 1 (got " + std::to_string(b) + ")");
  if (d < 1) throw invalid_argument("d must be positive (got " + std::to_string(d) + ")");
  if (kind < 0 || kind > 3)
    throw invalid_argument(
        "Invalid hash provided; hash must be one of `multiply shift', `multiply add shift', "
        "`tabulation8', or `tabulation16'");
  if (ilog2_int(b) > kMaxLog2B)
    throw unsupported("b = " + std::to_string(b) + " exceeds the largest supported b (2^24)");
  if (d > 65535) throw unsupported("d > 65535 is not supported");
}

static void check_sizes(int64_t n_a, int64_t n_inner, int64_t n_b) {
  if (n_a < 0 || n_inner < 0 || n_b < 0) throw invalid_argument("negative matrix dimension");
  if (n_a > 4294967296LL || n_b > 4294967296LL)
    throw unsupported("matrix dimensions above 2^32 exceed the u32 hash key range");
}

// ------------------------------------------------------------- pipeline
struct Codes {
  DevBuf a, b;  // d x n_a, d x n_b
};

static DevBuf upload(const void* h, size_t n, cudaStream_t s) {
  DevBuf d(n, s);
  if (n) CMM_CUDA(cudaMemcpyAsync(d.ptr, h, n, cudaMemcpyHostToDevice, s));
  return d;
}

// second per-thread, per-device stream for host-to-device row copies
static cudaStream_t copy_stream() {
  static thread_local std::map<int, cudaStream_t> streams;
  int dev = 0;
  CMM_CUDA(cudaGetDevice(&dev));
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t s;
  CMM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  streams[dev] = s;
  return s;
}

// Rows of AT and B (the inner index k) copied from host memory while the
// device works on earlier rows.  The host entry points allocate the device
// matrices and hand a feed to the sketch; its chunk loop calls wait() before
// the first use of rows [k0, k0 + c).  The copies run on copy_stream() in
// pieces of the sketch's chunk size, one event each, issued one piece ahead
// of the chunk being computed (pageable host memory is staged by host
// threads, host_to_device, while the previous chunk's kernels run).
class RowFeed {
 public:
  RowFeed(const void* hAT, const void* hB, void* dAT, void* dB, int64_t n_a, int64_t n_b,
          int64_t n_inner, size_t elem, cudaStream_t s)
      : hAT_(static_cast<const char*>(hAT)), hB_(static_cast<const char*>(hB)),
        dAT_(static_cast<char*>(dAT)), dB_(static_cast<char*>(dB)), rowA_((size_t)n_a * elem),
        rowB_((size_t)n_b * elem), n_inner_(n_inner), s_(s), cs_(copy_stream()) {
    cudaEvent_t ready;  // the device matrices are allocated on s
    CMM_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    CMM_CUDA(cudaEventRecord(ready, s));
    CMM_CUDA(cudaStreamWaitEvent(cs_, ready, 0));
    CMM_CUDA(cudaEventDestroy(ready));
  }
  RowFeed(const RowFeed&) = delete;
  RowFeed& operator=(const RowFeed&) = delete;
  // pieces still unwaited (an error ended the sketch early) are ordered
  // before s's later work, which frees the device matrices
  ~RowFeed() {
    for (auto& pc : pieces_) {
      if (!pc.waited) cudaStreamWaitEvent(s_, pc.ev, 0);
      cudaEventDestroy(pc.ev);
    }
  }
  // makes s wait until rows [0, k0 + c) are on the device; the first call
  // fixes the piece length to c
  void wait(int64_t k0, int64_t c, cudaStream_t s) {
    if (piece_ == 0) piece_ = c > 0 ? c : 1;
    const int64_t want = k0 + c + piece_ < n_inner_ ? k0 + c + piece_ : n_inner_;
    while (issued_ < want) issue();
    for (auto& pc : pieces_)
      if (!pc.waited && pc.k0 < k0 + c) {
        CMM_CUDA(cudaStreamWaitEvent(s, pc.ev, 0));
        pc.waited = true;
      }
  }
  void wait_all(cudaStream_t s) { wait(0, n_inner_, s); }

 private:
  struct Piece {
    int64_t k0;
    cudaEvent_t ev;
    bool waited;
  };
  void issue() {
    const int64_t k0 = issued_, c = n_inner_ - k0 < piece_ ? n_inner_ - k0 : piece_;
    if (rowA_) host_to_device(dAT_ + k0 * rowA_, hAT_ + k0 * rowA_, c * rowA_, cs_);
    if (rowB_) host_to_device(dB_ + k0 * rowB_, hB_ + k0 * rowB_, c * rowB_, cs_);
    Piece pc{k0, nullptr, false};
    CMM_CUDA(cudaEventCreateWithFlags(&pc.ev, cudaEventDisableTiming));
    CMM_CUDA(cudaEventRecord(pc.ev, cs_));
    pieces_.push_back(pc);
    issued_ = k0 + c;
  }
  const char* hAT_;
  const char* hB_;
  char* dAT_;
  char* dB_;
  size_t rowA_, rowB_;
  int64_t n_inner_, piece_ = 0, issued_ = 0;
  cudaStream_t s_, cs_;
  std::vector<Piece> pieces_;
};

// codes of both sides for keys 0..n_a-1 and 0..n_b-1
static Codes make_codes(const SketchParams& sp, int64_t n_a, int64_t n_b, cudaStream_t s) {
  DevBuf params = upload(sp.blob.data(), sp.blob.size(), s);
  const size_t set = sp.fn_bytes * (size_t)sp.d;
  const uint8_t* base = params.as<uint8_t>();
  Codes c;
  c.a = DevBuf((size_t)sp.d * (size_t)n_a * 4, s);
  c.b = DevBuf((size_t)sp.d * (size_t)n_b * 4, s);
  launch_hash_codes(sp.kind, base, base + 2 * set, sp.d, sp.log2b, n_a, c.a.as<uint32_t>(), s);
  launch_hash_codes(sp.kind, base + set, base + 3 * set, sp.d, sp.log2b, n_b, c.b.as<uint32_t>(), s);
  return c;
}

// Budget for the per-chunk materialized rows (d copies of each row pair).
// Bytes for the materialized rows of one chunk of inner indices: a third of
// the free device memory, at most 8 GiB, or CMM_MATERIALIZE_BYTES when set
// (smaller budgets run more chunks).
static size_t materialize_budget() {
  size_t free_b = 0, total_b = 0;
  CMM_CUDA(cudaMemGetInfo(&free_b, &total_b));
  size_t cap = (size_t)8 << 30;
  if (const char* e = getenv("CMM_MATERIALIZE_BYTES")) {
    const long long v = atoll(e);
    if (v > 0 && (size_t)v < cap) cap = (size_t)v;
  }
  return free_b / 3 < cap ? free_b / 3 : cap;
}

// The cluster kernels when this device can co-schedule a cluster of them
// and the residue segments fit in shared memory; false -> the slab kernels.
// CMM_SKETCH_KERNELS = cluster | slab forces one family where both apply
// (for comparisons); unset or "auto" takes the measured-faster choice.
static int sketch_kernel_choice() {
  static const int choice = [] {
    const char* e = getenv("CMM_SKETCH_KERNELS");
    if (e && !strcmp(e, "cluster")) return 1;
    if (e && !strcmp(e, "slab")) return 2;
    return 0;
  }();
  return choice;
}

static bool try_cluster_plan(int variant, bool f32, const Codes& codes, int64_t n_a, int64_t n_b,
                             int64_t n_inner, const SketchParams& sp, ClusterPlan& C, SlabPlan& plan,
                             cudaStream_t s) {
  if (!sketch_cluster_applicable(variant, f32, sp.b)) return false;
  if (sketch_kernel_choice() == 2) return false;
  // auto: measured on B200 at n = 16384, d = 9 -- the group kernels win
  // for every FFT case, for FP64 FWHT (86.6 against 176-188 ms of sketch
  // kernel per product at b = 2^16 on the slab kernel) and for FP32 FWHT
  // (351 against 509 ms at b = 2^18 on the tensor-core slab kernel)
  try {
    C = plan_cluster(variant, f32, n_inner, sp.d, sp.b, n_a, n_b);
  } catch (const unsupported&) {
    return false;
  }
  plan = make_residue_plan(codes.a.as<uint32_t>(), codes.b.as<uint32_t>(), n_a, n_b, sp.d, sp.b,
                           C.logL, C.logR2, s);
  return cluster_smem_fits(variant, f32, C, plan);
}

// Inner indices of the sketch chunk starting at k0.  While rows are still
// arriving from the host, the first chunk is an eighth of the budget, so the
// device starts after a short copy.
static int64_t chunk_len(int64_t k0, int64_t kc, int64_t n_inner, const RowFeed* feed) {
  const int64_t cmax = (feed && k0 == 0 && kc >= 64) ? kc / 8 : kc;
  return n_inner - k0 < cmax ? n_inner - k0 : cmax;
}

// feed != nullptr: the rows of dAT / dB are still arriving from the host;
// every chunk waits for its rows (and computes their FFT row scales) first.
static void sketch_device(int variant, const SketchParams& sp, const Codes& codes, int64_t n_a,
                          int64_t n_inner, int64_t n_b, const double* dAT, const double* dB,
                          double* dP, cudaStream_t s, RowFeed* feed = nullptr) {
  const double2* tw = twiddles(sp.b, s);
  const size_t elem = variant == kVariantFFT ? 16 : 8;
  DevBuf scale;
  if (variant == kVariantFFT) scale = DevBuf((size_t)(n_inner > 0 ? n_inner : 1) * 4, s);
  // rows [k0, k0 + c) usable on s: arrived, and scaled for the FFT
  auto rows_ready = [&](int64_t k0, int64_t c) {
    if (feed) feed->wait(k0, c, s);
    if (variant == kVariantFFT)
      launch_row_scale(dAT + k0 * n_a, dB + k0 * n_b, n_a, c, n_b, scale.as<int>() + k0, s);
  };
  ClusterPlan C;
  SlabPlan plan;
  if (n_inner > 0 && try_cluster_plan(variant, false, codes, n_a, n_b, n_inner, sp, C, plan, s)) {
    // residue plan + per-chunk materialized rows + cluster kernels
    set_sketch_kernel("cluster");
    const int64_t SA = plan.slots_a(), SB = plan.slots_b();
    const size_t per_row = (size_t)sp.d * (size_t)(SA + SB) * 8;
    int64_t kc = (int64_t)(materialize_budget() / per_row);
    if (kc < 1) kc = 1;
    if (kc > n_inner) kc = n_inner;
    DevBuf matA((size_t)sp.d * kc * SA * 8, s), matB((size_t)sp.d * kc * SB * 8, s);
    DevBuf partial((size_t)C.G * sp.d * (size_t)sp.b * elem, s);
    for (int64_t k0 = 0, c = 0; k0 < n_inner; k0 += c) {
      c = chunk_len(k0, kc, n_inner, feed);
      rows_ready(k0, c);
      launch_materialize(plan, dAT, dB, k0, c, matA.as<double>(), matB.as<double>(), s);
      launch_sketch_cluster(variant, false, C, plan, matA.ptr, matB.ptr, c, scale.as<int>(), k0, tw,
                            partial.ptr, sp.d, k0 > 0 ? 1 : 0, s);
    }
    DevBuf work(2 * (size_t)sp.d * (size_t)sp.b * 16, s);
    launch_finalize_natural(variant, sp.d, sp.b, C.G, partial.ptr, tw, work.ptr, dP, s);
    return;
  }
  if (n_inner > 0 && sketch_v1_applicable(variant, sp.b, n_a, n_b)) {
    // bucket-sorted plan + per-chunk materialized rows + v1 kernels
    set_sketch_kernel("slab");
    const SketchPlan P = plan_sketch_v1(variant, n_a, n_inner, n_b, sp.d, sp.b, num_sms());
    SlabPlan plan = make_slab_plan(codes.a.as<uint32_t>(), codes.b.as<uint32_t>(), n_a, n_b, sp.d,
                                   sp.b, P.logL, s);
    const int64_t SA = (int64_t)plan.EA * kPlanThreads, SB = (int64_t)plan.EB * kPlanThreads;
    const size_t per_row = (size_t)sp.d * (size_t)(SA + SB) * 8;
    int64_t kc = (int64_t)(materialize_budget() / per_row);
    if (kc < 1) kc = 1;
    if (kc > n_inner) kc = n_inner;
    DevBuf matA((size_t)sp.d * kc * SA * 8, s), matB((size_t)sp.d * kc * SB * 8, s);
    DevBuf partial((size_t)P.G * sp.d * (size_t)sp.b * elem, s);
    for (int64_t k0 = 0, c = 0; k0 < n_inner; k0 += c) {
      c = chunk_len(k0, kc, n_inner, feed);
      rows_ready(k0, c);
      launch_materialize(plan, dAT, dB, k0, c, matA.as<double>(), matB.as<double>(), s);
      launch_sketch_v1(P, plan, matA.as<double>(), matB.as<double>(), c, scale.as<int>(), k0, tw,
                       partial.ptr, k0 > 0 ? 1 : 0, s);
    }
    DevBuf work(2 * (size_t)sp.d * (size_t)sp.b * 16, s);
    launch_finalize(P, partial.ptr, tw, work.ptr, dP, s);
    return;
  }
  const SketchPlan P = plan_sketch(variant, n_a, n_inner, n_b, sp.d, sp.b, num_sms());
  set_sketch_kernel("small-b");
  rows_ready(0, n_inner);
  DevBuf partial((size_t)P.G * sp.d * (size_t)sp.b * elem, s);
  launch_sketch_accumulate(P, dAT, dB, codes.a.as<uint32_t>(), codes.b.as<uint32_t>(),
                           scale.as<int>(), tw, partial.ptr, s);
  DevBuf work(2 * (size_t)sp.d * (size_t)sp.b * 16, s);
  launch_finalize(P, partial.ptr, tw, work.ptr, dP, s);
}

// Mixed-precision compressed product from FP32 inputs.  Slabs of 8192 on
// the FP32 kernels when b >= 8192; smaller b runs the FP64 kernels on an
// FP64 copy of the inputs (on the device).
static void sketch_device_mixed(int variant, const SketchParams& sp, const Codes& codes,
                                int64_t n_a, int64_t n_inner, int64_t n_b, const float* dAT,
                                const float* dB, double* dP, cudaStream_t s,
                                RowFeed* feed = nullptr) {
  if (!(n_inner > 0 && sketch_mixed_applicable(variant, sp.b))) {
    if (feed) feed->wait_all(s);
    DevBuf A64((size_t)n_inner * n_a * 8, s), B64((size_t)n_inner * n_b * 8, s);
    launch_f32_to_f64(dAT, A64.as<double>(), n_inner * n_a, s);
    launch_f32_to_f64(dB, B64.as<double>(), n_inner * n_b, s);
    sketch_device(variant, sp, codes, n_a, n_inner, n_b, A64.as<double>(), B64.as<double>(), dP, s);
    return;
  }
  const double2* tw = twiddles(sp.b, s);
  const size_t elem = variant == kVariantFFT ? 16 : 8;
  DevBuf scale((size_t)n_inner * 4, s);
  auto rows_ready = [&](int64_t k0, int64_t c) {
    if (feed) feed->wait(k0, c, s);
    if (variant == kVariantFFT)
      launch_row_scale_f32(dAT + k0 * n_a, dB + k0 * n_b, n_a, c, n_b, scale.as<int>() + k0, s);
  };
  ClusterPlan Cp;
  SlabPlan cplan;
  if (try_cluster_plan(variant, true, codes, n_a, n_b, n_inner, sp, Cp, cplan, s)) {
    set_sketch_kernel("cluster");
    SlabPlan& plan = cplan;
    const int64_t SA = plan.slots_a(), SB = plan.slots_b();
    const size_t per_row = (size_t)sp.d * (size_t)(SA + SB) * 4;
    int64_t kc = (int64_t)(materialize_budget() / per_row);
    if (kc < 1) kc = 1;
    if (kc > n_inner) kc = n_inner;
    DevBuf matA((size_t)sp.d * kc * SA * 4, s), matB((size_t)sp.d * kc * SB * 4, s);
    DevBuf partial((size_t)Cp.G * sp.d * (size_t)sp.b * elem, s);
    for (int64_t k0 = 0, c = 0; k0 < n_inner; k0 += c) {
      c = chunk_len(k0, kc, n_inner, feed);
      rows_ready(k0, c);
      launch_materialize_f32(plan, dAT, dB, k0, c, matA.as<float>(), matB.as<float>(), s);
      launch_sketch_cluster(variant, true, Cp, plan, matA.ptr, matB.ptr, c, scale.as<int>(), k0, tw,
                            partial.ptr, sp.d, k0 > 0 ? 1 : 0, s);
    }
    DevBuf work(2 * (size_t)sp.d * (size_t)sp.b * 16, s);
    launch_finalize_natural(variant, sp.d, sp.b, Cp.G, partial.ptr, tw, work.ptr, dP, s);
    return;
  }
  const SketchPlan P = plan_sketch_mixed(variant, n_a, n_inner, n_b, sp.d, sp.b, num_sms());
  set_sketch_kernel("slab-mixed");
  SlabPlan plan = make_slab_plan(codes.a.as<uint32_t>(), codes.b.as<uint32_t>(), n_a, n_b, sp.d,
                                 sp.b, P.logL, s);
  const int64_t SA = (int64_t)plan.EA * kPlanThreads, SB = (int64_t)plan.EB * kPlanThreads;
  const size_t per_row = (size_t)sp.d * (size_t)(SA + SB) * 4;
  int64_t kc = (int64_t)(materialize_budget() / per_row);
  if (kc < 1) kc = 1;
  if (kc > n_inner) kc = n_inner;
  DevBuf matA((size_t)sp.d * kc * SA * 4, s), matB((size_t)sp.d * kc * SB * 4, s);
  DevBuf partial((size_t)P.G * sp.d * (size_t)sp.b * elem, s);
  for (int64_t k0 = 0, c = 0; k0 < n_inner; k0 += c) {
    c = chunk_len(k0, kc, n_inner, feed);
    rows_ready(k0, c);
    launch_materialize_f32(plan, dAT, dB, k0, c, matA.as<float>(), matB.as<float>(), s);
    launch_sketch_mixed(P, plan, matA.as<float>(), matB.as<float>(), c, scale.as<int>(), k0, tw,
                        partial.ptr, k0 > 0 ? 1 : 0, s);
  }
  DevBuf work(2 * (size_t)sp.d * (size_t)sp.b * 16, s);
  launch_finalize(P, partial.ptr, tw, work.ptr, dP, s);
}

static uint64_t pick_seed(int has_seed, uint64_t seed) { return has_seed ? seed : time_seed(); }

// The dense estimate comes back to the host in row blocks: every block's
// decompression is enqueued on s first, then each block's copy on
// copy_stream() after its event, so the copies overlap the decompression of
// the later blocks (pageable host memory: each block is drained through the
// staging slots, device_to_host, while later blocks decompress).  Returns
// when C is on the host.
// a synchronous entry point reports a group barrier wait that ran out
static void check_group_waits() {
  if (sketch_group_timed_out())
    throw std::runtime_error("cluster sketch: a group barrier wait ran out; the sketch is invalid");
}

static void decompress_to_host(int variant, int d, int b, int64_t n_a, int64_t n_b, const Codes& codes,
                               const double* dP, double* dC, double* C, cudaStream_t s) {
  struct Join {  // s waits for the copies before anything later (frees) runs on it
    cudaStream_t s, cs;
    std::vector<cudaEvent_t> ev;
    ~Join() {
      cudaEvent_t done;
      if (cudaEventCreateWithFlags(&done, cudaEventDisableTiming) == cudaSuccess) {
        cudaEventRecord(done, cs);
        cudaStreamWaitEvent(s, done, 0);
        cudaEventDestroy(done);
      }
      for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
  } join{s, copy_stream(), {}};
  if (n_a > 0 && n_b > 0) {
    int64_t rows = (n_a + 7) / 8;
    rows = (rows + 15) / 16 * 16;
    for (int64_t i0 = 0; i0 < n_a; i0 += rows) {
      const int64_t r = n_a - i0 < rows ? n_a - i0 : rows;
      launch_decompress_dense_rows(variant, d, b, n_a, n_b, i0, r, codes.a.as<uint32_t>(), codes.b.as<uint32_t>(),
                                   dP, dC + i0 * n_b, s);
      cudaEvent_t e;
      CMM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      join.ev.push_back(e);
      CMM_CUDA(cudaEventRecord(e, s));
    }
    size_t blk = 0;
    for (int64_t i0 = 0; i0 < n_a; i0 += rows, ++blk) {
      const int64_t r = n_a - i0 < rows ? n_a - i0 : rows;
      CMM_CUDA(cudaStreamWaitEvent(join.cs, join.ev[blk], 0));
      device_to_host(C + i0 * n_b, dC + i0 * n_b, (size_t)r * n_b * 8, join.cs);
    }
  }
  CMM_CUDA(cudaStreamSynchronize(join.cs));
  CMM_CUDA(cudaStreamSynchronize(s));
  check_group_waits();
}

// ------------------------------------------------------- instrumentation
static std::atomic<int64_t> g_launches{0};
static std::atomic<bool> g_prof{false};
static std::mutex g_prof_mu;
struct FamilyTimes {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  cudaEvent_t open = nullptr;
};
static std::map<std::string, FamilyTimes>& prof_table() {
  static std::map<std::string, FamilyTimes> t;
  return t;
}

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

static thread_local std::string g_sketch_kernel;
void set_sketch_kernel(const char* name) { g_sketch_kernel = name; }

bool prof_set(bool on) { return g_prof.exchange(on); }

void prof_begin(const char* family, cudaStream_t s) {
  if (!g_prof.load()) return;
  std::lock_guard<std::mutex> g(g_prof_mu);
  FamilyTimes& f = prof_table()[family];
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, s);
  f.open = e;
}

void prof_end(const char* family, cudaStream_t s) {
  if (!g_prof.load()) return;
  std::lock_guard<std::mutex> g(g_prof_mu);
  FamilyTimes& f = prof_table()[family];
  if (!f.open) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, s);
  f.ev.emplace_back(f.open, e);
  f.open = nullptr;
}

}  // namespace cmm

// ================================================================= C ABI
using namespace cmm;

template <typename F>
static int guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return CMM_OK;
  } catch (const cmm::invalid_argument& e) {
    g_last_error = e.what();
    return CMM_ERR_INVALID_ARGUMENT;
  } catch (const cmm::unsupported& e) {
    g_last_error = e.what();
    return CMM_ERR_UNSUPPORTED;
  } catch (const cmm::cuda_error& e) {
    g_last_error = e.what();
    return CMM_ERR_CUDA;
  } catch (const std::bad_alloc&) {
    g_last_error = "out of memory";
    return CMM_ERR_NO_MEMORY;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return CMM_ERR_RUNTIME;
  } catch (...) {
    g_last_error = "unknown error";
    return CMM_ERR_RUNTIME;
  }
}

extern "C" {

const char* cmm_last_error(void) { return g_last_error.c_str(); }

const char* cmm_version(void) { return "compmatmul_b200 0.1.0 (sm_100a)"; }

int cmm_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int cmm_max_buckets(void) { return 1 << kMaxLog2B; }

void cmm_profile_enable(int on) { g_prof.store(on != 0); }

void cmm_profile_reset(void) {
  std::lock_guard<std::mutex> g(g_prof_mu);
  for (auto& kv : prof_table()) {
    for (auto& pr : kv.second.ev) {
      cudaEventSynchronize(pr.second);
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
    if (kv.second.open) cudaEventDestroy(kv.second.open);
  }
  prof_table().clear();
}

int cmm_profile_read(const char* family, double* total_ms, int64_t* launches) {
  return guarded([&] {
    std::lock_guard<std::mutex> g(g_prof_mu);
    double tot = 0.0;
    int64_t n = 0;
    auto it = prof_table().find(family ? family : "");
    if (it != prof_table().end()) {
      for (auto& pr : it->second.ev) {
        CMM_CUDA(cudaEventSynchronize(pr.second));
        float ms = 0.f;
        CMM_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
        tot += ms;
        ++n;
      }
    }
    if (total_ms) *total_ms = tot;
    if (launches) *launches = n;
  });
}

int64_t cmm_launch_count(void) { return g_launches.load(); }

const char* cmm_last_sketch_kernel(void) { return g_sketch_kernel.c_str(); }

int cmm_batch_create(const cmm_batch_product* products, int count, int f32, int tune, void** handle) {
  return guarded([&] {
    if (!handle) throw invalid_argument("handle must not be null");
    *handle = nullptr;
    *handle = batch_create(products, count, f32 != 0, tune != 0);
  });
}

int cmm_batch_run(void* handle, void* stream) {
  return guarded([&] { batch_run(static_cast<BatchPlan*>(handle), (cudaStream_t)stream); });
}

int cmm_batch_info(void* handle, int64_t* items, int* ctas, int* launches) {
  return guarded([&] { batch_info(static_cast<const BatchPlan*>(handle), items, ctas, launches); });
}

int cmm_batch_config(void* handle, int product, int* log2_slab, int* radix, int* groups, int* tuned) {
  return guarded(
      [&] { batch_config(static_cast<const BatchPlan*>(handle), product, log2_slab, radix, groups, tuned); });
}

int cmm_batch_destroy(void* handle) {
  return guarded([&] { batch_destroy(static_cast<BatchPlan*>(handle)); });
}

int cmm_server_create(const cmm_server_config* cfg, void** server) {
  return guarded([&] {
    if (!server) throw invalid_argument("server must not be null");
    *server = nullptr;
    *server = server_create(cfg);
  });
}

int cmm_server_submit(void* server, const cmm_request* req, uint64_t* id) {
  return guarded([&] {
    const uint64_t v = server_submit(static_cast<Server*>(server), req);
    if (id) *id = v;
  });
}

int cmm_server_wait(void* server, uint64_t id, double timeout_s, int* done, double* latency_s) {
  return guarded([&] {
    const bool d = server_wait(static_cast<Server*>(server), id, timeout_s, latency_s);
    if (done) *done = d ? 1 : 0;
  });
}

int cmm_server_stats_get(void* server, cmm_server_stats* out) {
  return guarded([&] { server_stats(static_cast<Server*>(server), out); });
}

int cmm_server_destroy(void* server) {
  return guarded([&] { server_destroy(static_cast<Server*>(server)); });
}

int cmm_cluster_phase_cycles(double* cycles, double* steps) {
  return guarded([&] {
    if (!cluster_phase_cycles(cycles, steps))
      throw unsupported("built without CMM_PHASE_CLOCKS (set CMM_EXTRA_NVFLAGS=-DCMM_PHASE_CLOCKS and rebuild)");
  });
}

int cmm_probe_fma_tflops(int fp64, double* tflops) {
  return guarded([&] {
    if (!tflops) throw invalid_argument("tflops must not be null");
    *tflops = probe_fma_tflops(fp64 != 0, host_stream());
  });
}

int cmm_dev_compressed_product(int variant, int hash_kind, int64_t n_a, int64_t n_inner,
                               int64_t n_b, const double* dAT, const double* dB, int d, int b,
                               uint64_t seed, double* dP, void* stream) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    check_sizes(n_a, n_inner, n_b);
    cudaStream_t s = (cudaStream_t)stream;
    SketchParams sp = make_sketch_params(hash_kind, d, b, seed);
    Codes codes = make_codes(sp, n_a, n_b, s);
    sketch_device(variant, sp, codes, n_a, n_inner, n_b, dAT, dB, dP, s);
  });
}

// Allocation-free twin of cmm_dev_compressed_product: the slab pipeline
// (hash codes -> row balance -> k_sketch_{fft,fwht} -> k-group reduction +
// inverse) with every intermediate carved from the static device scratch.
// The sizes are checked against the scratch before any CUDA call.
int cmm_dev_compressed_product_noalloc(int variant, int hash_kind, int64_t n_a, int64_t n_inner,
                                       int64_t n_b, const double* dAT, const double* dB, int d,
                                       int b, uint64_t seed, double* dP, void* stream) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    check_sizes(n_a, n_inner, n_b);
    const bool fft = variant == kVariantFFT;
    const size_t elem = fft ? 16 : 8;
    const size_t db = (size_t)d * (size_t)b;
    auto a256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t off = 0;
    auto take = [&](size_t n) { const size_t o = off; off += a256(n); return o; };
    const size_t set = hash_param_bytes(hash_kind) * (size_t)d;
    const size_t o_blob = take(4 * set);
    const size_t o_ca = take((size_t)d * (size_t)n_a * 4);
    const size_t o_cb = take((size_t)d * (size_t)n_b * 4);
    const size_t o_scale = take(fft ? (size_t)(n_inner > 0 ? n_inner : 1) * 4 : 0);
    const size_t o_tw = take((size_t)b * 16);
    const size_t o_work = take(2 * db * elem);
    const size_t o_part = off;
    if (o_part > kNoAllocScratchBytes || kNoAllocScratchBytes - o_part < db * elem)
      throw unsupported("cmm_dev_compressed_product_noalloc: this product needs " +
                        std::to_string(o_part + db * elem) + " bytes of scratch; the static scratch holds " +
                        std::to_string(kNoAllocScratchBytes) +
                        " bytes (use cmm_dev_compressed_product for larger sizes)");
    const int64_t g_fit = (int64_t)((kNoAllocScratchBytes - o_part) / (db * elem));

    cudaStream_t s = (cudaStream_t)stream;
    SketchPlan P = plan_sketch(variant, n_a, n_inner, n_b, d, b, num_sms());
    if (P.G > g_fit) P.G = (int)g_fit;
    uint8_t* base = static_cast<uint8_t*>(noalloc_scratch());
    const SketchParams sp = make_sketch_params(hash_kind, d, b, seed);
    CMM_CUDA(cudaMemcpyAsync(base + o_blob, sp.blob.data(), sp.blob.size(), cudaMemcpyHostToDevice, s));
    uint32_t* ca = reinterpret_cast<uint32_t*>(base + o_ca);
    uint32_t* cb = reinterpret_cast<uint32_t*>(base + o_cb);
    launch_hash_codes(hash_kind, base + o_blob, base + o_blob + 2 * set, d, sp.log2b, n_a, ca, s);
    launch_hash_codes(hash_kind, base + o_blob + set, base + o_blob + 3 * set, d, sp.log2b, n_b, cb, s);
    // w[j] = exp(-2 pi i j / b): the process-wide host table (built once per b)
    CMM_CUDA(cudaMemcpyAsync(base + o_tw, host_twiddles(b).data(), sizeof(double2) * (size_t)b,
                             cudaMemcpyHostToDevice, s));
    const double2* tw = reinterpret_cast<const double2*>(base + o_tw);
    int* scale = fft ? reinterpret_cast<int*>(base + o_scale) : nullptr;
    if (fft) launch_row_scale(dAT, dB, n_a, n_inner, n_b, scale, s);
    void* part = base + o_part;
    CMM_CUDA(cudaMemsetAsync(part, 0, (size_t)P.G * db * elem, s));  // k-group partials start at zero
    launch_sketch_accumulate(P, dAT, dB, ca, cb, scale, tw, part, s);
    launch_finalize(P, part, tw, base + o_work, dP, s);
  });
}

int cmm_dev_decompress_dense(int variant, int hash_kind, int64_t n_a, int64_t n_b, int d, int b,
                             uint64_t seed, const double* dP, double* dC, void* stream) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    check_sizes(n_a, 0, n_b);
    cudaStream_t s = (cudaStream_t)stream;
    SketchParams sp = make_sketch_params(hash_kind, d, b, seed);
    Codes codes = make_codes(sp, n_a, n_b, s);
    launch_decompress_dense(variant, d, b, n_a, n_b, codes.a.as<uint32_t>(), codes.b.as<uint32_t>(),
                            dP, dC, s);
  });
}

int cmm_dev_matmul(int variant, int hash_kind, int64_t n_a, int64_t n_inner, int64_t n_b,
                   double* dC, const double* dAT, const double* dB, int d, int b, uint64_t seed,
                   void* stream) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    check_sizes(n_a, n_inner, n_b);
    cudaStream_t s = (cudaStream_t)stream;
    SketchParams sp = make_sketch_params(hash_kind, d, b, seed);
    Codes codes = make_codes(sp, n_a, n_b, s);
    DevBuf P((size_t)d * (size_t)b * 8, s);
    sketch_device(variant, sp, codes, n_a, n_inner, n_b, dAT, dB, P.as<double>(), s);
    launch_decompress_dense(variant, d, b, n_a, n_b, codes.a.as<uint32_t>(), codes.b.as<uint32_t>(),
                            P.as<double>(), dC, s);
  });
}

int cmm_dev_topk(const double* dC, int64_t n_a, int64_t n_b, int K, uint32_t* d_i, uint32_t* d_j,
                 double* d_v, void* stream) {
  return guarded([&] {
    if (n_a < 0 || n_b < 0 || K < 0) throw cmm::invalid_argument("negative size");
    topk_dense(dC, n_a, n_b, K, d_i, d_j, d_v, (cudaStream_t)stream);
  });
}

int cmm_dev_decompress_entries(int variant, int hash_kind, int d, int b, uint64_t seed, const double* dP,
                               int64_t count, const uint32_t* dI, const uint32_t* dJ, double* dOut,
                               void* stream) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    if (count < 0) throw cmm::invalid_argument("negative count");
    if (count == 0) return;
    cudaStream_t s = (cudaStream_t)stream;
    SketchParams sp = make_sketch_params(hash_kind, d, b, seed);
    DevBuf params = upload(sp.blob.data(), sp.blob.size(), s);
    const size_t set = sp.fn_bytes * (size_t)d;
    const uint8_t* base = params.as<uint8_t>();
    DevBuf cI((size_t)d * count * 4, s), cJ((size_t)d * count * 4, s);
    launch_hash_codes_keys(hash_kind, base, base + 2 * set, d, sp.log2b, count, dI, cI.as<uint32_t>(), s);
    launch_hash_codes_keys(hash_kind, base + set, base + 3 * set, d, sp.log2b, count, dJ, cJ.as<uint32_t>(), s);
    launch_decompress_list(variant, d, b, count, cI.as<uint32_t>(), cJ.as<uint32_t>(), dP, dOut, s);
  });
}

int cmm_dev_sketch_topk(int variant, int hash_kind, int64_t n_a, int64_t n_b, int d, int b, uint64_t seed,
                        const double* dP, int K, size_t scratch_bytes, uint32_t* d_i, uint32_t* d_j, double* d_v,
                        void* stream) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    check_sizes(n_a, 0, n_b);
    if (K < 0) throw cmm::invalid_argument("negative K");
    if (K == 0) return;
    if ((int64_t)K > n_a * n_b) throw cmm::invalid_argument("K exceeds the number of entries");
    cudaStream_t s = (cudaStream_t)stream;
    if (scratch_bytes == 0) scratch_bytes = (size_t)256 << 20;
    // rows per tile: the tile's dense estimate fits the scratch and holds >= K entries
    int64_t rows = (int64_t)(scratch_bytes / (8 * (size_t)n_b));
    rows = std::max<int64_t>(rows, ((int64_t)K + n_b - 1) / n_b);
    rows = std::min<int64_t>(std::max<int64_t>(rows, 1), n_a);
    SketchParams sp = make_sketch_params(hash_kind, d, b, seed);
    DevBuf params = upload(sp.blob.data(), sp.blob.size(), s);
    const size_t set = sp.fn_bytes * (size_t)d;
    const uint8_t* base = params.as<uint8_t>();
    DevBuf cB((size_t)d * (size_t)n_b * 4, s);
    launch_hash_codes(hash_kind, base + set, base + 3 * set, d, sp.log2b, n_b, cB.as<uint32_t>(), s);
    DevBuf tile((size_t)rows * (size_t)n_b * 8, s), keys((size_t)rows * 4, s), cA((size_t)d * (size_t)rows * 4, s);
    DevBuf ti((size_t)K * 4, s), tj((size_t)K * 4, s), tv((size_t)K * 8, s);
    struct Cand { double v; uint64_t idx; };
    std::vector<Cand> cand;
    std::vector<uint32_t> hi((size_t)K), hj((size_t)K), hk((size_t)rows);
    std::vector<double> hv((size_t)K);
    for (int64_t i0 = 0; i0 < n_a; i0 += rows) {
      const int64_t r = std::min<int64_t>(rows, n_a - i0);
      for (int64_t e = 0; e < r; ++e) hk[(size_t)e] = (uint32_t)(i0 + e);
      CMM_CUDA(cudaMemcpyAsync(keys.ptr, hk.data(), (size_t)r * 4, cudaMemcpyHostToDevice, s));
      launch_hash_codes_keys(hash_kind, base, base + 2 * set, d, sp.log2b, r, keys.as<uint32_t>(),
                             cA.as<uint32_t>(), s);
      launch_decompress_dense(variant, d, b, r, n_b, cA.as<uint32_t>(), cB.as<uint32_t>(), dP, tile.as<double>(), s);
      const int kt = (int)std::min<int64_t>(K, r * n_b);
      topk_dense(tile.as<double>(), r, n_b, kt, ti.as<uint32_t>(), tj.as<uint32_t>(), tv.as<double>(), s);
      CMM_CUDA(cudaMemcpyAsync(hi.data(), ti.ptr, (size_t)kt * 4, cudaMemcpyDeviceToHost, s));
      CMM_CUDA(cudaMemcpyAsync(hj.data(), tj.ptr, (size_t)kt * 4, cudaMemcpyDeviceToHost, s));
      CMM_CUDA(cudaMemcpyAsync(hv.data(), tv.ptr, (size_t)kt * 8, cudaMemcpyDeviceToHost, s));
      CMM_CUDA(cudaStreamSynchronize(s));
      for (int e = 0; e < kt; ++e)
        cand.push_back({hv[(size_t)e], (uint64_t)(i0 + hi[(size_t)e]) * (uint64_t)n_b + hj[(size_t)e]});
    }
    // the tiles' top-K lists contain the global top-K under the same order:
    // value descending (the device order of the bit keys), then (i, j)
    auto key = [](double v) {
      uint64_t b;
      std::memcpy(&b, &v, 8);
      return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
    };
    std::sort(cand.begin(), cand.end(), [&](const Cand& a, const Cand& c) {
      const uint64_t ka = key(a.v), kc = key(c.v);
      return ka != kc ? ka > kc : a.idx < c.idx;
    });
    for (int e = 0; e < K; ++e) {
      hi[(size_t)e] = (uint32_t)(cand[(size_t)e].idx / (uint64_t)n_b);
      hj[(size_t)e] = (uint32_t)(cand[(size_t)e].idx % (uint64_t)n_b);
      hv[(size_t)e] = cand[(size_t)e].v;
    }
    CMM_CUDA(cudaMemcpyAsync(d_i, hi.data(), (size_t)K * 4, cudaMemcpyHostToDevice, s));
    CMM_CUDA(cudaMemcpyAsync(d_j, hj.data(), (size_t)K * 4, cudaMemcpyHostToDevice, s));
    CMM_CUDA(cudaMemcpyAsync(d_v, hv.data(), (size_t)K * 8, cudaMemcpyHostToDevice, s));
    CMM_CUDA(cudaStreamSynchronize(s));
  });
}

int cmm_dev_gemm(int64_t n_a, int64_t n_inner, int64_t n_b, double* dC, const double* dAT,
                 const double* dB, void* stream) {
  return guarded([&] {
    check_sizes(n_a, n_inner, n_b);
    launch_gemm(n_a, n_inner, n_b, dC, dAT, dB, (cudaStream_t)stream);
  });
}

int cmm_dev_compressed_product_f32(int variant, int hash_kind, int64_t n_a, int64_t n_inner,
                                   int64_t n_b, const float* dAT, const float* dB, int d, int b,
                                   uint64_t seed, double* dP, void* stream) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    check_sizes(n_a, n_inner, n_b);
    cudaStream_t s = (cudaStream_t)stream;
    SketchParams sp = make_sketch_params(hash_kind, d, b, seed);
    Codes codes = make_codes(sp, n_a, n_b, s);
    sketch_device_mixed(variant, sp, codes, n_a, n_inner, n_b, dAT, dB, dP, s);
  });
}

int cmm_dev_matmul_f32(int variant, int hash_kind, int64_t n_a, int64_t n_inner, int64_t n_b,
                       double* dC, const float* dAT, const float* dB, int d, int b, uint64_t seed,
                       void* stream) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    check_sizes(n_a, n_inner, n_b);
    cudaStream_t s = (cudaStream_t)stream;
    SketchParams sp = make_sketch_params(hash_kind, d, b, seed);
    Codes codes = make_codes(sp, n_a, n_b, s);
    DevBuf P((size_t)d * (size_t)b * 8, s);
    sketch_device_mixed(variant, sp, codes, n_a, n_inner, n_b, dAT, dB, P.as<double>(), s);
    launch_decompress_dense(variant, d, b, n_a, n_b, codes.a.as<uint32_t>(), codes.b.as<uint32_t>(),
                            P.as<double>(), dC, s);
  });
}

int cmm_compressed_product_f32(int variant, int hash_kind, int64_t n_a, int64_t n_inner,
                               int64_t n_b, const float* AT, const float* B, int d, int b,
                               int has_seed, uint64_t seed, double* p_out, uint64_t* seed_out) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    check_sizes(n_a, n_inner, n_b);
    const uint64_t sd = pick_seed(has_seed, seed);
    if (seed_out) *seed_out = sd;
    cudaStream_t s = host_stream();
    DevBuf dAT((size_t)n_inner * n_a * 4, s), dB((size_t)n_inner * n_b * 4, s);
    RowFeed feed(AT, B, dAT.ptr, dB.ptr, n_a, n_b, n_inner, 4, s);
    SketchParams sp = make_sketch_params(hash_kind, d, b, sd);
    Codes codes = make_codes(sp, n_a, n_b, s);
    DevBuf P((size_t)d * (size_t)b * 8, s);
    sketch_device_mixed(variant, sp, codes, n_a, n_inner, n_b, dAT.as<float>(), dB.as<float>(),
                        P.as<double>(), s, &feed);
    CMM_CUDA(cudaMemcpyAsync(p_out, P.ptr, P.bytes, cudaMemcpyDeviceToHost, s));
    CMM_CUDA(cudaStreamSynchronize(s));
    check_group_waits();
  });
}

int cmm_matmul_f32(int variant, int hash_kind, int64_t n_a, int64_t n_inner, int64_t n_b,
                   double* C, const float* AT, const float* B, int d, int b, int has_seed,
                   uint64_t seed) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    check_sizes(n_a, n_inner, n_b);
    const uint64_t sd = pick_seed(has_seed, seed);
    cudaStream_t s = host_stream();
    DevBuf dAT((size_t)n_inner * n_a * 4, s), dB((size_t)n_inner * n_b * 4, s);
    RowFeed feed(AT, B, dAT.ptr, dB.ptr, n_a, n_b, n_inner, 4, s);
    DevBuf dC((size_t)n_a * n_b * 8, s);
    SketchParams sp = make_sketch_params(hash_kind, d, b, sd);
    Codes codes = make_codes(sp, n_a, n_b, s);
    DevBuf P((size_t)d * (size_t)b * 8, s);
    sketch_device_mixed(variant, sp, codes, n_a, n_inner, n_b, dAT.as<float>(), dB.as<float>(),
                        P.as<double>(), s, &feed);
    decompress_to_host(variant, d, b, n_a, n_b, codes, P.as<double>(), dC.as<double>(), C, s);
  });
}

int cmm_dev_wht_rows_f32(const float* x, float* y, int64_t rows, int log2n, int method, void* stream) {
  return guarded([&] { wht_rows_f32(x, y, rows, log2n, method, (cudaStream_t)stream); });
}

int cmm_compressed_product(int variant, int hash_kind, int64_t n_a, int64_t n_inner, int64_t n_b,
                           const double* AT, const double* B, int d, int b, int has_seed,
                           uint64_t seed, double* p_out, uint64_t* seed_out) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    check_sizes(n_a, n_inner, n_b);
    const uint64_t sd = pick_seed(has_seed, seed);
    if (seed_out) *seed_out = sd;
    cudaStream_t s = host_stream();
    DevBuf dAT((size_t)n_inner * n_a * 8, s), dB((size_t)n_inner * n_b * 8, s);
    RowFeed feed(AT, B, dAT.ptr, dB.ptr, n_a, n_b, n_inner, 8, s);
    SketchParams sp = make_sketch_params(hash_kind, d, b, sd);
    Codes codes = make_codes(sp, n_a, n_b, s);
    DevBuf P((size_t)d * (size_t)b * 8, s);
    sketch_device(variant, sp, codes, n_a, n_inner, n_b, dAT.as<double>(), dB.as<double>(),
                  P.as<double>(), s, &feed);
    CMM_CUDA(cudaMemcpyAsync(p_out, P.ptr, P.bytes, cudaMemcpyDeviceToHost, s));
    CMM_CUDA(cudaStreamSynchronize(s));
    check_group_waits();
  });
}

int cmm_matmul(int variant, int hash_kind, int64_t n_a, int64_t n_inner, int64_t n_b, double* C,
               const double* AT, const double* B, int d, int b, int has_seed, uint64_t seed) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    check_sizes(n_a, n_inner, n_b);
    const uint64_t sd = pick_seed(has_seed, seed);
    cudaStream_t s = host_stream();
    DevBuf dAT((size_t)n_inner * n_a * 8, s), dB((size_t)n_inner * n_b * 8, s);
    RowFeed feed(AT, B, dAT.ptr, dB.ptr, n_a, n_b, n_inner, 8, s);
    DevBuf dC((size_t)n_a * n_b * 8, s);
    SketchParams sp = make_sketch_params(hash_kind, d, b, sd);
    Codes codes = make_codes(sp, n_a, n_b, s);
    DevBuf P((size_t)d * (size_t)b * 8, s);
    sketch_device(variant, sp, codes, n_a, n_inner, n_b, dAT.as<double>(), dB.as<double>(),
                  P.as<double>(), s, &feed);
    decompress_to_host(variant, d, b, n_a, n_b, codes, P.as<double>(), dC.as<double>(), C, s);
  });
}

int cmm_decompress(int variant, int hash_kind, int d, int b, uint64_t seed, const double* p,
                   int64_t count, const uint32_t* i, const uint32_t* j, double* out) {
  return guarded([&] {
    check_params(variant, hash_kind, d, b);
    if (count < 0) throw cmm::invalid_argument("negative count");
    if (count == 0) return;
    cudaStream_t s = host_stream();
    SketchParams sp = make_sketch_params(hash_kind, d, b, seed);
    DevBuf params = upload(sp.blob.data(), sp.blob.size(), s);
    const size_t set = sp.fn_bytes * (size_t)d;
    const uint8_t* base = params.as<uint8_t>();
    DevBuf dI = upload(i, (size_t)count * 4, s), dJ = upload(j, (size_t)count * 4, s);
    DevBuf cI((size_t)d * count * 4, s), cJ((size_t)d * count * 4, s);
    launch_hash_codes_keys(hash_kind, base, base + 2 * set, d, sp.log2b, count, dI.as<uint32_t>(),
                           cI.as<uint32_t>(), s);
    launch_hash_codes_keys(hash_kind, base + set, base + 3 * set, d, sp.log2b, count,
                           dJ.as<uint32_t>(), cJ.as<uint32_t>(), s);
    DevBuf dP = upload(p, (size_t)d * b * 8, s);
    DevBuf dOut((size_t)count * 8, s);
    launch_decompress_list(variant, d, b, count, cI.as<uint32_t>(), cJ.as<uint32_t>(),
                           dP.as<double>(), dOut.as<double>(), s);
    CMM_CUDA(cudaMemcpyAsync(out, dOut.ptr, dOut.bytes, cudaMemcpyDeviceToHost, s));
    CMM_CUDA(cudaStreamSynchronize(s));
  });
}

int cmm_gemm(int64_t n_a, int64_t n_inner, int64_t n_b, double* C, const double* AT,
             const double* B) {
  return guarded([&] {
    check_sizes(n_a, n_inner, n_b);
    cudaStream_t s = host_stream();
    DevBuf dAT = upload(AT, (size_t)n_inner * n_a * 8, s);
    DevBuf dB = upload(B, (size_t)n_inner * n_b * 8, s);
    DevBuf dC((size_t)n_a * n_b * 8, s);
    launch_gemm(n_a, n_inner, n_b, dC.as<double>(), dAT.as<double>(), dB.as<double>(), s);
    if (dC.bytes) CMM_CUDA(cudaMemcpyAsync(C, dC.ptr, dC.bytes, cudaMemcpyDeviceToHost, s));
    CMM_CUDA(cudaStreamSynchronize(s));
  });
}

int cmm_hash_codes(int hash_kind, int d, int b, uint64_t seed, int side, int64_t n,
                   uint32_t* codes_out) {
  return guarded([&] {
    check_params(kVariantFFT, hash_kind, d, b);
    if (side != 0 && side != 1) throw cmm::invalid_argument("side must be 0 or 1");
    if (n < 0) throw cmm::invalid_argument("negative n");
    if (n == 0) return;
    cudaStream_t s = host_stream();
    SketchParams sp = make_sketch_params(hash_kind, d, b, seed);
    DevBuf params = upload(sp.blob.data(), sp.blob.size(), s);
    const size_t set = sp.fn_bytes * (size_t)d;
    const uint8_t* base = params.as<uint8_t>();
    DevBuf c((size_t)d * n * 4, s);
    launch_hash_codes(hash_kind, base + side * set, base + (2 + side) * set, d, sp.log2b, n,
                      c.as<uint32_t>(), s);
    CMM_CUDA(cudaMemcpyAsync(codes_out, c.ptr, c.bytes, cudaMemcpyDeviceToHost, s));
    CMM_CUDA(cudaStreamSynchronize(s));
  });
}

// --------------------------------------------- host-side rng and hash draws
// No CUDA call: these give C++ callers of the header entry points the
// reference's rng and hash objects (rng.hpp, hashing.hpp) bit for bit.

void cmm_rng_seed(uint64_t seed, uint64_t* state) {
  const Xoshiro256ss r(seed);
  for (int i = 0; i < 4; ++i) state[i] = r.s[i];
}

uint64_t cmm_rng_next(uint64_t* state) {
  Xoshiro256ss r(0);
  for (int i = 0; i < 4; ++i) r.s[i] = state[i];
  const uint64_t v = r();
  for (int i = 0; i < 4; ++i) state[i] = r.s[i];
  return v;
}

uint64_t cmm_time_millis(void) { return time_millis(); }

int cmm_hash_params(int hash_kind, int n, uint64_t buckets, uint64_t seed, void* out, size_t out_bytes) {
  return guarded([&] {
    if (hash_kind < 0 || hash_kind > 3) throw cmm::invalid_argument("unknown hash kind");
    if (buckets == 0 || (buckets & (buckets - 1)) != 0)
      throw cmm::invalid_argument("The number of buckets must be a power of 2");
    if (n < 0) throw cmm::invalid_argument("negative function count");
    const size_t need = hash_param_bytes(hash_kind) * (size_t)n;
    if (out_bytes < need)
      throw cmm::invalid_argument("output buffer holds " + std::to_string(out_bytes) + " bytes, " +
                                  std::to_string(need) + " needed");
    if (n == 0) return;
    const std::vector<uint8_t> v = draw_hash_params(hash_kind, n, seed);
    std::memcpy(out, v.data(), need);
  });
}

}  // extern "C"
