// Serving engine: continuous batching of independent compressed products.
//
// A scheduler thread owns the device work.  Submitted requests wait in
// arrival order; a request is admitted when the device bytes it needs fit
// under the cap next to those of the requests already admitted.  Admission
// enqueues its preparation on the upload stream (input copy, hash codes,
// row balance, sorted plan).  Whenever a compute stream is free, the admitted
// requests that are not yet running -- at most max_wave of them -- form a
// wave: one persistent k_batch_sketch launch over all of their work items,
// then each request's k-group reduction + inverse and the copy of its
// sketch to pinned staging.  Waves on different streams overlap on the
// device, so requests that arrive while others run start as soon as memory
// and a stream free up.  A finished wave releases its requests' memory and
// copies each sketch to the caller's buffer.
//
// A request's k-groups, hence its work items and every summation order,
// follow from the request alone (never from the wave it runs in), so a
// result is bit-identical alone and in any mix.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "cmm_batch.h"

namespace cmm {
namespace {

using Clock = std::chrono::steady_clock;

// pinned host blocks reused by size class (powers of two from 64 KB)
class PinnedPool {
 public:
  ~PinnedPool() {
    for (auto& kv : free_)
      for (void* p : kv.second) cudaFreeHost(p);
  }
  void* get(size_t n, size_t* cls) {
    size_t c = 65536;
    while (c < n) c <<= 1;
    *cls = c;
    auto& v = free_[c];
    if (!v.empty()) {
      void* p = v.back();
      v.pop_back();
      return p;
    }
    void* p = nullptr;
    CMM_CUDA(cudaMallocHost(&p, c));
    return p;
  }
  void put(void* p, size_t cls) { free_[cls].push_back(p); }

 private:
  std::map<size_t, std::vector<void*>> free_;
};

// hash codes and sorted plan of one (hash, seed, d, b, n_a, n_b, slab):
// fixed by those alone, shared read-only by every request that has them
struct CodePlan {
  DevBuf params, codes_a, codes_b;
  SlabPlan plan;
  size_t bytes = 0;
};
using CodeKey = std::tuple<int, uint64_t, int, int, int64_t, int64_t, int>;

struct Request {
  uint64_t id = 0;
  cmm_request r{};
  Clock::time_point t_submit, t_done;
  size_t need = 0;
  int log2b = 0, logL = 0, radix = 8, tc = 1, G = 1;
  bool done = false;
  std::string error;
  // device state (allocated on the upload stream at admission)
  DevBuf in_a, in_b, scale, partial, p_dev, work;
  std::shared_ptr<CodePlan> cp;  // codes + plan (cached or this request's own)
  SketchPlan sp{};
  const double2* tw = nullptr;
  cudaEvent_t prepared = nullptr;
  void* stage = nullptr;  // pinned copy of p
  size_t stage_cls = 0;
};

struct Wave {
  std::vector<std::shared_ptr<Request>> reqs;
  int stream = 0;
  DevBuf dprods, counter;  // dprods: products | items | finalize jobs
  void* host = nullptr;      // pinned staging of those tables
  size_t host_cls = 0;
  cudaEvent_t done = nullptr;
};

size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }
int ilog2i(int64_t x) {
  int l = 0;
  while (((int64_t)1 << l) < x) ++l;
  return l;
}

}  // namespace

struct Server {
  cmm_server_config cfg{};
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> incoming;
  std::map<uint64_t, std::shared_ptr<Request>> by_id;
  uint64_t next_id = 1;
  size_t mem_in_use = 0, max_mem = 0;
  cmm_server_stats stats{};
  std::string error;  // sticky scheduler failure
  bool stop = false;
  // scheduler-thread state
  std::vector<std::shared_ptr<Request>> ready;  // admitted, not yet in a wave
  std::vector<std::unique_ptr<Wave>> waves;
  std::vector<cudaStream_t> streams;
  std::vector<bool> busy;
  cudaStream_t up = nullptr;
  int ctas = 0;
  const double2* tw4096 = nullptr;
  PinnedPool pinned;
  std::thread th;
  // residency of hash codes + plans (scheduler thread only), LRU order
  std::map<CodeKey, std::pair<std::shared_ptr<CodePlan>, uint64_t>> cache;
  uint64_t cache_clock = 0;
  size_t cache_bytes = 0;
};

namespace {

// shape-dependent parts of a request; identical for a request alone and in
// any mix
void geometry(Request& q, bool f32) {
  const cmm_request& r = q.r;
  q.log2b = ilog2i(r.b);
  const int lmax = r.variant == kVariantFFT ? kBatchFftLog : kBatchWhtLog;
  int logL = std::min(q.log2b, lmax), radix = 8, tc = 1;
  int tl = 0, tr = 0, tt = 1;
  if (batch_tuned(r.variant, f32, q.log2b, r.n_a + r.n_b, &tl, &tr, &tt)) {
    logL = tl;
    radix = tr;
    tc = tt;
  }
  q.logL = logL;
  q.radix = radix;
  q.tc = tc;
  // items of about the cost of 64 rows of a 2048 + 2048 product at L = 4096
  const double target = 64.0 * batch_unit_cost(2048, 2048, 12);
  const double row = batch_unit_cost(r.n_a, r.n_b, logL);
  int64_t G = (int64_t)std::ceil((double)r.n_inner * row / target);
  G = std::max<int64_t>(1, std::min<int64_t>({G, std::max<int64_t>(1, r.n_inner / 8), 65535}));
  q.G = (int)G;
  SketchPlan& P = q.sp;
  P = SketchPlan{};
  P.variant = r.variant;
  P.d = r.d;
  P.b = r.b;
  P.log2b = q.log2b;
  P.logL = logL;
  P.L = 1 << logL;
  P.logR = q.log2b - logL;
  P.R = 1 << P.logR;
  P.KB = 1;
  P.G = q.G;
  P.n_a = r.n_a;
  P.n_inner = r.n_inner;
  P.n_b = r.n_b;
  // device bytes held while admitted
  const size_t esz = f32 ? 4 : 8, elem = r.variant == kVariantFFT ? 16 : 8;
  const size_t d = (size_t)r.d, nab = (size_t)(r.n_a + r.n_b);
  const size_t sa = (size_t)std::max<int64_t>(r.n_a, 8), sb = (size_t)std::max<int64_t>(r.n_b, 8);
  const size_t cb = q.log2b <= 16 ? 2 : 4;
  size_t need = 0;
  if (!r.inputs_on_device) need += round256(esz * (size_t)r.n_inner * (size_t)r.n_a) + round256(esz * (size_t)r.n_inner * (size_t)r.n_b);
  need += round256(4 * hash_param_bytes(r.hash_kind) * d);
  need += round256(4 * d * (size_t)std::max<int64_t>(r.n_a, 1)) + round256(4 * d * (size_t)std::max<int64_t>(r.n_b, 1));
  need += round256(4 * (size_t)std::max<int64_t>(r.n_inner, 1));
  need += 2 * round256(d * (sa + sb) * (4 + cb)) + round256(2 * d * 513 * 4) * 2;  // plan + its sort scratch
  need += round256(4 * d * nab);                                                    // sort scratch
  need += round256((size_t)q.G * d * (size_t)r.b * elem);
  need += round256(d * (size_t)r.b * 8) + round256(2 * d * (size_t)r.b * 16);
  q.need = need;
}

void prepare(Server& S, Request& q) {
  const cmm_request& r = q.r;
  const bool f32 = S.cfg.f32 != 0;
  const size_t esz = f32 ? 4 : 8, elem = r.variant == kVariantFFT ? 16 : 8;
  cudaStream_t s = S.up;
  const void* AT = r.AT;
  const void* B = r.B;
  if (!r.inputs_on_device && r.n_inner > 0) {
    q.in_a = DevBuf(esz * (size_t)r.n_inner * (size_t)r.n_a, s);
    q.in_b = DevBuf(esz * (size_t)r.n_inner * (size_t)r.n_b, s);
    if (q.in_a.bytes) CMM_CUDA(cudaMemcpyAsync(q.in_a.ptr, r.AT, q.in_a.bytes, cudaMemcpyHostToDevice, s));
    if (q.in_b.bytes) CMM_CUDA(cudaMemcpyAsync(q.in_b.ptr, r.B, q.in_b.bytes, cudaMemcpyHostToDevice, s));
    AT = q.in_a.ptr;
    B = q.in_b.ptr;
  }
  // hash codes + sorted plan: from the residency cache, or built here
  const CodeKey key{r.hash_kind, r.seed, r.d, r.b, r.n_a, r.n_b, q.logL};
  auto hit = S.cache.find(key);
  if (hit != S.cache.end()) {
    q.cp = hit->second.first;
    hit->second.second = ++S.cache_clock;
    std::lock_guard<std::mutex> g(S.mu);
    S.stats.cache_hits += 1;
  } else {
    auto cp = std::make_shared<CodePlan>();
    const SketchParams sp = make_sketch_params(r.hash_kind, r.d, r.b, r.seed);
    cp->params = DevBuf(sp.blob.size(), s);
    CMM_CUDA(cudaMemcpyAsync(cp->params.ptr, sp.blob.data(), sp.blob.size(), cudaMemcpyHostToDevice, s));
    const size_t set = sp.fn_bytes * (size_t)r.d;
    const uint8_t* base = cp->params.as<uint8_t>();
    cp->codes_a = DevBuf(4 * (size_t)r.d * (size_t)std::max<int64_t>(r.n_a, 1), s);
    cp->codes_b = DevBuf(4 * (size_t)r.d * (size_t)std::max<int64_t>(r.n_b, 1), s);
    launch_hash_codes(r.hash_kind, base, base + 2 * set, r.d, q.log2b, r.n_a, cp->codes_a.as<uint32_t>(), s);
    launch_hash_codes(r.hash_kind, base + set, base + 3 * set, r.d, q.log2b, r.n_b, cp->codes_b.as<uint32_t>(), s);
    cp->plan = make_residue_plan(cp->codes_a.as<uint32_t>(), cp->codes_b.as<uint32_t>(), r.n_a, r.n_b, r.d, r.b,
                                 q.logL, 0, s);
    cp->bytes = cp->params.bytes + cp->codes_a.bytes + cp->codes_b.bytes + cp->plan.srcA.bytes + cp->plan.srcB.bytes +
                cp->plan.codeA.bytes + cp->plan.codeB.bytes + cp->plan.countA.bytes + cp->plan.countB.bytes;
    q.cp = cp;
    {
      std::lock_guard<std::mutex> g(S.mu);
      S.stats.cache_misses += 1;
    }
    if (S.cfg.cache_bytes > 0 && cp->bytes <= S.cfg.cache_bytes) {
      while (S.cache_bytes + cp->bytes > S.cfg.cache_bytes && !S.cache.empty()) {  // evict least recent
        auto lru = S.cache.begin();
        for (auto it = S.cache.begin(); it != S.cache.end(); ++it)
          if (it->second.second < lru->second.second) lru = it;
        S.cache_bytes -= lru->second.first->bytes;
        S.cache.erase(lru);  // in-flight requests keep their own reference
      }
      S.cache[key] = {cp, ++S.cache_clock};
      S.cache_bytes += cp->bytes;
    }
  }
  q.scale = DevBuf(4 * (size_t)std::max<int64_t>(r.n_inner, 1), s);
  if (r.variant == kVariantFFT && r.n_inner > 0) {
    if (f32) launch_row_scale_f32((const float*)AT, (const float*)B, r.n_a, r.n_inner, r.n_b, q.scale.as<int>(), s);
    else launch_row_scale((const double*)AT, (const double*)B, r.n_a, r.n_inner, r.n_b, q.scale.as<int>(), s);
  }
  q.partial = DevBuf((size_t)q.G * r.d * (size_t)r.b * elem, s);
  CMM_CUDA(cudaMemsetAsync(q.partial.ptr, 0, q.partial.bytes, s));  // k-groups without rows stay zero
  q.p_dev = DevBuf((size_t)r.d * (size_t)r.b * 8, s);
  q.work = DevBuf(2 * (size_t)r.d * (size_t)r.b * 16, s);
  q.tw = twiddles(r.b, s);
  q.r.AT = AT;  // device inputs from here on
  q.r.B = B;
  CMM_CUDA(cudaEventCreateWithFlags(&q.prepared, cudaEventDisableTiming));
  CMM_CUDA(cudaEventRecord(q.prepared, s));
  q.stage = S.pinned.get((size_t)r.d * (size_t)r.b * 8, &q.stage_cls);
}

BProd bprod(const Request& q) {
  BProd d{};
  d.AT = q.r.AT;
  d.B = q.r.B;
  const SlabPlan& pl = q.cp->plan;
  d.srcA = pl.srcA.as<uint32_t>();
  d.srcB = pl.srcB.as<uint32_t>();
  d.codeA = pl.codeA.ptr;
  d.codeB = pl.codeB.ptr;
  d.cutA = pl.countA.as<uint32_t>();
  d.cutB = pl.countB.as<uint32_t>();
  d.SA = pl.EA;
  d.SB = pl.EB;
  d.code16 = pl.u16 ? 1 : 0;
  d.scale = q.scale.as<int>();
  d.tw = q.tw;
  d.partial = q.partial.ptr;
  d.n_a = q.r.n_a;
  d.n_inner = q.r.n_inner;
  d.n_b = q.r.n_b;
  d.d = q.r.d;
  d.log2b = q.log2b;
  d.logL = q.logL;
  d.logR = q.log2b - q.logL;
  d.G = q.G;
  d.variant = q.r.variant;
  d.radix = q.radix;
  d.tc = q.tc;
  return d;
}

void launch_wave(Server& S, std::vector<std::shared_ptr<Request>> reqs, int si) {
  std::unique_ptr<Wave> W(new Wave());
  W->stream = si;
  cudaStream_t s = S.streams[(size_t)si];
  std::vector<BProd> prods;
  struct C { double c; BItem it; };
  std::vector<C> items;
  for (size_t i = 0; i < reqs.size(); ++i) {
    Request& q = *reqs[i];
    CMM_CUDA(cudaStreamWaitEvent(s, q.prepared, 0));
    prods.push_back(bprod(q));
    if (q.r.n_inner == 0) continue;
    const int64_t per = (q.r.n_inner + q.G - 1) / q.G;
    const double row = batch_unit_cost(q.r.n_a, q.r.n_b, q.logL);
    for (int64_t g = 0; g < q.G; ++g) {
      const int64_t rows = std::min<int64_t>(per, q.r.n_inner - g * per);
      if (rows <= 0) continue;
      for (int t = 0; t < q.r.d; ++t)
        for (int r = 0; r < (1 << (q.log2b - q.logL)); ++r) items.push_back({(double)rows * row, {(int)i, t, r, (int)g}});
    }
  }
  std::stable_sort(items.begin(), items.end(), [](const C& a, const C& b) { return a.c > b.c; });
  std::vector<FinJob> fin;  // one batched reduction + inverse for the small-b requests
  for (auto& qp : reqs)
    if (batch_finalize_fits(qp->log2b))
      for (int t = 0; t < qp->r.d; ++t)
        fin.push_back({qp->partial.ptr, qp->p_dev.as<double>(), qp->tw, qp->G, qp->r.d, t, qp->log2b, qp->logL,
                       qp->r.variant});
  // one pinned staging block and one device table: products | items | finalize jobs
  const size_t pb = prods.size() * sizeof(BProd), ib = items.size() * sizeof(BItem), fb = fin.size() * sizeof(FinJob);
  const size_t ioff = (pb + 15) & ~(size_t)15, foff = (ioff + ib + 15) & ~(size_t)15, total = foff + fb;
  W->host = S.pinned.get(std::max<size_t>(total, 16), &W->host_cls);
  unsigned char* hb = static_cast<unsigned char*>(W->host);
  std::memcpy(hb, prods.data(), pb);
  BItem* hi = reinterpret_cast<BItem*>(hb + ioff);
  for (size_t i = 0; i < items.size(); ++i) hi[i] = items[i].it;
  if (fb) std::memcpy(hb + foff, fin.data(), fb);
  W->dprods = DevBuf(std::max<size_t>(total, 16), s);
  W->counter = DevBuf(sizeof(int), s);
  CMM_CUDA(cudaMemcpyAsync(W->dprods.ptr, hb, total, cudaMemcpyHostToDevice, s));
  unsigned char* db = W->dprods.as<unsigned char>();
  const int n_items = (int)items.size();
  batch_launch_sketch(S.cfg.f32 != 0, reinterpret_cast<const BProd*>(db), reinterpret_cast<const BItem*>(db + ioff),
                      n_items, W->counter.as<int>(), S.tw4096, std::max(1, std::min(S.ctas, n_items)), s);
  batch_launch_finalize(reinterpret_cast<const FinJob*>(db + foff), (int)fin.size(), s);
  for (auto& qp : reqs) {
    Request& q = *qp;
    if (!batch_finalize_fits(q.log2b)) launch_finalize(q.sp, q.partial.ptr, q.tw, q.work.ptr, q.p_dev.as<double>(), s);
    CMM_CUDA(cudaMemcpyAsync(q.stage, q.p_dev.ptr, q.p_dev.bytes, cudaMemcpyDeviceToHost, s));
  }
  CMM_CUDA(cudaEventCreateWithFlags(&W->done, cudaEventDisableTiming));
  CMM_CUDA(cudaEventRecord(W->done, s));
  W->reqs = std::move(reqs);
  S.busy[(size_t)si] = true;
  {
    std::lock_guard<std::mutex> g(S.mu);
    S.stats.waves += 1;
    S.waves.push_back(std::move(W));
    S.stats.max_waves_in_flight = std::max<int64_t>(S.stats.max_waves_in_flight, (int64_t)S.waves.size());
  }
}

void finish_wave(Server& S, std::unique_ptr<Wave>& W) {
  const auto now = Clock::now();
  for (auto& qp : W->reqs) {
    Request& q = *qp;
    std::memcpy(q.r.p, q.stage, (size_t)q.r.d * (size_t)q.r.b * 8);
    S.pinned.put(q.stage, q.stage_cls);
    q.stage = nullptr;
    cudaEventDestroy(q.prepared);
    q.prepared = nullptr;
    // device buffers return to the pool (their work has completed)
    q.in_a = DevBuf();
    q.in_b = DevBuf();
    q.scale = DevBuf();
    q.partial = DevBuf();
    q.p_dev = DevBuf();
    q.work = DevBuf();
    q.cp.reset();  // a cached plan stays resident for later requests
    q.t_done = now;
  }
  S.pinned.put(W->host, W->host_cls);
  cudaEventDestroy(W->done);
  S.busy[(size_t)W->stream] = false;
  {
    std::lock_guard<std::mutex> g(S.mu);
    for (auto& qp : W->reqs) {
      qp->done = true;
      S.mem_in_use -= qp->need;
      S.stats.completed += 1;
      S.stats.in_flight -= 1;
    }
  }
  S.cv_done.notify_all();
}

void fail_all(Server& S, const std::string& msg) {
  std::lock_guard<std::mutex> g(S.mu);
  S.error = msg;
  for (auto& kv : S.by_id)
    if (!kv.second->done) {
      kv.second->done = true;
      kv.second->error = msg;
    }
  S.cv_done.notify_all();
}

void scheduler(Server* Sp) {
  Server& S = *Sp;
  try {
    CMM_CUDA(cudaSetDevice(S.device));
    for (;;) {
      bool progress = false;
      // completions (in launch order per stream is not required: poll all)
      for (size_t i = 0; i < S.waves.size();) {
        const cudaError_t e = cudaEventQuery(S.waves[i]->done);
        if (e == cudaSuccess) {
          finish_wave(S, S.waves[i]);
          std::lock_guard<std::mutex> g(S.mu);
          S.waves.erase(S.waves.begin() + (long)i);
          progress = true;
        } else if (e == cudaErrorNotReady) {
          ++i;
        } else {
          CMM_CUDA(e);
        }
      }
      // admission in arrival order, bounded by the memory cap
      std::vector<std::shared_ptr<Request>> admit;
      {
        std::lock_guard<std::mutex> g(S.mu);
        while (!S.incoming.empty() && S.mem_in_use + S.incoming.front()->need <= S.cfg.mem_cap_bytes) {
          auto q = S.incoming.front();
          S.incoming.pop_front();
          S.mem_in_use += q->need;
          S.max_mem = std::max(S.max_mem, S.mem_in_use);
          S.stats.queued -= 1;
          S.stats.in_flight += 1;
          admit.push_back(q);
        }
      }
      for (auto& q : admit) {
        prepare(S, *q);
        S.ready.push_back(q);
        progress = true;
      }
      // waves: every free stream takes up to max_wave ready requests
      for (size_t si = 0; si < S.streams.size() && !S.ready.empty(); ++si) {
        if (S.busy[si]) continue;
        const size_t n = std::min<size_t>(S.ready.size(), (size_t)S.cfg.max_wave);
        std::vector<std::shared_ptr<Request>> w(S.ready.begin(), S.ready.begin() + (long)n);
        S.ready.erase(S.ready.begin(), S.ready.begin() + (long)n);
        launch_wave(S, std::move(w), (int)si);
        progress = true;
      }
      if (!progress) {
        std::unique_lock<std::mutex> lk(S.mu);
        if (S.stop && S.incoming.empty() && S.ready.empty() && S.waves.empty()) break;
        S.cv_work.wait_for(lk, std::chrono::microseconds(S.waves.empty() ? 2000 : 50));
      }
    }
  } catch (const std::exception& e) {
    fail_all(S, e.what());
  } catch (...) {
    fail_all(S, "serving scheduler failed");
  }
}

}  // namespace

Server* server_create(const cmm_server_config* cfg) {
  if (!cfg) throw invalid_argument("config must not be null");
  if (cfg->streams < 1 || cfg->streams > 64) throw invalid_argument("streams must be in [1, 64]");
  if (cfg->max_wave < 1) throw invalid_argument("max_wave must be positive");
  if (cfg->mem_cap_bytes < ((size_t)1 << 20)) throw invalid_argument("mem_cap_bytes must be at least 1 MiB");
  std::unique_ptr<Server> S(new Server());
  S->cfg = *cfg;
  CMM_CUDA(cudaGetDevice(&S->device));
  CMM_CUDA(cudaStreamCreateWithFlags(&S->up, cudaStreamNonBlocking));
  for (int i = 0; i < cfg->streams; ++i) {
    cudaStream_t s;
    CMM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    S->streams.push_back(s);
    S->busy.push_back(false);
  }
  S->ctas = batch_resident_ctas(cfg->f32 != 0);
  S->tw4096 = twiddles(1 << kBatchFftLog, S->up);
  // map the admission cap into the stream-ordered pool once, so that
  // admissions do not grow the pool while requests run (the pool keeps
  // freed memory); less when the device has less free memory
  {
    { DevBuf first(256, S->up); }  // sets the pool to keep freed memory
    size_t free_b = 0, total_b = 0;
    CMM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    size_t want = std::min(cfg->mem_cap_bytes + cfg->cache_bytes, free_b / 10 * 9);
    while (want >= ((size_t)64 << 20)) {
      void* p = nullptr;
      if (cudaMallocAsync(&p, want, S->up) == cudaSuccess) {
        CMM_CUDA(cudaFreeAsync(p, S->up));
        break;
      }
      cudaGetLastError();
      want /= 2;
    }
    CMM_CUDA(cudaStreamSynchronize(S->up));
  }
  S->th = std::thread(scheduler, S.get());
  return S.release();
}

uint64_t server_submit(Server* S, const cmm_request* req) {
  if (!S) throw invalid_argument("server handle is null");
  if (!req) throw invalid_argument("request must not be null");
  const cmm_request& r = *req;
  if (r.variant != kVariantFFT && r.variant != kVariantFWHT) throw invalid_argument("invalid variant");
  if (r.b < 2 || (r.b & (r.b - 1)) != 0)
    throw invalid_argument("b must be power of 2 greater than 1 (got " + std::to_string(r.b) + ")");
  if (r.d < 1) throw invalid_argument("d must be positive (got " + std::to_string(r.d) + ")");
  if (r.hash_kind < 0 || r.hash_kind > 3)
    throw invalid_argument("Invalid hash provided; hash must be one of `multiply shift', `multiply add shift', "
                           "`tabulation8', or `tabulation16'");
  if (ilog2i(r.b) > kMaxLog2B) throw unsupported("b exceeds the largest supported b (2^24)");
  if (r.d > 65535) throw unsupported("d > 65535 is not supported");
  if (r.n_a < 0 || r.n_inner < 0 || r.n_b < 0) throw invalid_argument("negative matrix dimension");
  if (r.n_a > 4294967296LL || r.n_b > 4294967296LL) throw unsupported("dimension above 2^32");
  if (r.n_inner > 0 && ((r.n_a > 0 && !r.AT) || (r.n_b > 0 && !r.B))) throw invalid_argument("AT or B is null");
  if (!r.p) throw invalid_argument("p is null");
  auto q = std::make_shared<Request>();
  q->r = r;
  geometry(*q, S->cfg.f32 != 0);
  if (q->need > S->cfg.mem_cap_bytes)
    throw invalid_argument("request needs " + std::to_string(q->need) + " device bytes, above the admission cap of " +
                           std::to_string(S->cfg.mem_cap_bytes));
  std::lock_guard<std::mutex> g(S->mu);
  if (!S->error.empty()) throw runtime_error("server failed: " + S->error);
  if (S->stop) throw runtime_error("server is stopping");
  q->id = S->next_id++;
  q->t_submit = Clock::now();
  S->incoming.push_back(q);
  S->by_id[q->id] = q;
  S->stats.submitted += 1;
  S->stats.queued += 1;
  S->cv_work.notify_one();
  return q->id;
}

bool server_wait(Server* S, uint64_t id, double timeout_s, double* latency_s) {
  if (!S) throw invalid_argument("server handle is null");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->by_id.find(id);
  if (it == S->by_id.end()) throw invalid_argument("unknown request id " + std::to_string(id));
  std::shared_ptr<Request> q = it->second;
  auto pred = [&] { return q->done; };
  if (timeout_s < 0) S->cv_done.wait(lk, pred);
  else S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred);
  if (!q->done) return false;
  if (!q->error.empty()) throw runtime_error("request failed: " + q->error);
  if (latency_s) *latency_s = std::chrono::duration<double>(q->t_done - q->t_submit).count();
  return true;
}

void server_stats(Server* S, cmm_server_stats* out) {
  if (!S) throw invalid_argument("server handle is null");
  if (!out) throw invalid_argument("stats must not be null");
  std::lock_guard<std::mutex> g(S->mu);
  *out = S->stats;
  out->mem_in_use = S->mem_in_use;
  out->max_mem_in_use = S->max_mem;
  out->cache_in_use = S->cache_bytes;
}

void server_destroy(Server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->th.joinable()) S->th.join();
  std::string err;
  {
    std::lock_guard<std::mutex> g(S->mu);
    err = S->error;
    S->by_id.clear();
    S->cache.clear();
  }
  cudaStreamSynchronize(S->up);
  for (cudaStream_t s : S->streams) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  cudaStream_t up = S->up;
  delete S;  // pinned pool and remaining buffers
  cudaStreamSynchronize(up);
  cudaStreamDestroy(up);
  if (!err.empty()) throw runtime_error("server failed: " + err);
}

}  // namespace cmm
