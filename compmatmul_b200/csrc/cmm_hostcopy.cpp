// Copies between device memory and caller-owned host memory for the
// host-pointer entry points (the drop-in's matmul_fft / matmul_fwht pass
// ordinary pageable numpy arrays, compmatmul.cpp:107-147).
//
// Page-locked host memory is copied directly with cudaMemcpyAsync.  For
// pageable memory the driver stages the copy through its own pinned buffer
// on one host thread, well below the link's bandwidth; here it goes through
// a ring of pinned slots that several host threads fill (host to device) or
// drain (device to host) at once, while the DMA of the previous slot runs.
#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "cmm_internal.h"

namespace cmm {
namespace {

// memcpy split over a small persistent pool of host threads
class CopyPool {
 public:
  static CopyPool& get() {
    static CopyPool* pool = new CopyPool();  // lives until exit (threads detach)
    return *pool;
  }

  void copy(void* dst, const void* src, size_t n) {
    constexpr size_t kMinPart = (size_t)4 << 20;
    const size_t parts = std::min<size_t>(workers_.size() + 1, (n + kMinPart - 1) / kMinPart);
    if (parts <= 1) {
      std::memcpy(dst, src, n);
      return;
    }
    const size_t part = (n + parts - 1) / parts;
    Latch latch;
    latch.left = parts - 1;
    {
      std::lock_guard<std::mutex> g(mu_);
      for (size_t p = 1; p < parts; ++p) {
        const size_t off = p * part;
        jobs_.push_back({static_cast<char*>(dst) + off, static_cast<const char*>(src) + off,
                         std::min(part, n - off), &latch});
      }
    }
    cv_.notify_all();
    std::memcpy(dst, src, std::min(part, n));
    std::unique_lock<std::mutex> lk(latch.mu);
    latch.cv.wait(lk, [&] { return latch.left == 0; });
  }

 private:
  struct Latch {
    std::mutex mu;
    std::condition_variable cv;
    size_t left = 0;
  };
  struct Job {
    char* dst;
    const char* src;
    size_t n;
    Latch* latch;
  };

  CopyPool() {
    const unsigned hw = std::thread::hardware_concurrency();
    const unsigned n = hw > 1 ? std::min(hw, 16u) - 1 : 0;
    for (unsigned i = 0; i < n; ++i) {
      workers_.emplace_back([this] { run(); });
      workers_.back().detach();
    }
  }

  void run() {
    for (;;) {
      Job j;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !jobs_.empty(); });
        j = jobs_.front();
        jobs_.pop_front();
      }
      std::memcpy(j.dst, j.src, j.n);
      std::lock_guard<std::mutex> g(j.latch->mu);
      if (--j.latch->left == 0) j.latch->cv.notify_all();
    }
  }

  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<Job> jobs_;
};

// Pinned staging slots of one host thread on one device: each slot's event
// marks the end of the last copy that used it.
class Staging {
 public:
  static constexpr int kSlots = 4;
  static constexpr size_t kSlotBytes = (size_t)64 << 20;

  static Staging& get() {
    static thread_local std::map<int, Staging> per_device;
    int dev = 0;
    CMM_CUDA(cudaGetDevice(&dev));
    return per_device[dev];
  }

  Staging() = default;
  Staging(const Staging&) = delete;
  Staging& operator=(const Staging&) = delete;
  ~Staging() {
    for (int i = 0; i < kSlots; ++i) {
      if (ev_[i]) cudaEventDestroy(ev_[i]);
      if (buf_[i]) cudaFreeHost(buf_[i]);
    }
  }

  // slot i, free for host access (its last copy has completed)
  char* slot(int i) {
    if (!buf_[i]) {
      CMM_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&buf_[i]), kSlotBytes, cudaHostAllocDefault));
      CMM_CUDA(cudaEventCreateWithFlags(&ev_[i], cudaEventDisableTiming));
    } else {
      CMM_CUDA(cudaEventSynchronize(ev_[i]));
    }
    return buf_[i];
  }
  cudaEvent_t event(int i) { return ev_[i]; }
  int next() {
    const int i = next_;
    next_ = (next_ + 1) % kSlots;
    return i;
  }

 private:
  char* buf_[kSlots] = {};
  cudaEvent_t ev_[kSlots] = {};
  int next_ = 0;
};

bool pageable(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

}  // namespace

void host_to_device(void* dst, const void* src, size_t bytes, cudaStream_t cs) {
  if (bytes == 0) return;
  if (!pageable(src)) {
    CMM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, cs));
    return;
  }
  Staging& st = Staging::get();
  for (size_t off = 0; off < bytes; off += Staging::kSlotBytes) {
    const size_t n = std::min(Staging::kSlotBytes, bytes - off);
    const int i = st.next();
    char* s = st.slot(i);
    CopyPool::get().copy(s, static_cast<const char*>(src) + off, n);
    CMM_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + off, s, n, cudaMemcpyHostToDevice, cs));
    CMM_CUDA(cudaEventRecord(st.event(i), cs));
  }
}

void device_to_host(void* dst, const void* src, size_t bytes, cudaStream_t cs) {
  if (bytes == 0) return;
  if (!pageable(dst)) {
    CMM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, cs));
    return;
  }
  // the DMA of up to kSlots pieces is in flight while the host drains the
  // oldest one
  Staging& st = Staging::get();
  struct Piece {
    size_t off, n;
    int slot;
    char* buf;
  };
  std::deque<Piece> inflight;
  auto drain = [&] {
    const Piece p = inflight.front();
    inflight.pop_front();
    CMM_CUDA(cudaEventSynchronize(st.event(p.slot)));
    CopyPool::get().copy(static_cast<char*>(dst) + p.off, p.buf, p.n);
  };
  for (size_t off = 0; off < bytes; off += Staging::kSlotBytes) {
    if ((int)inflight.size() == Staging::kSlots) drain();
    const size_t n = std::min(Staging::kSlotBytes, bytes - off);
    const int i = st.next();
    char* s = st.slot(i);
    CMM_CUDA(cudaMemcpyAsync(s, static_cast<const char*>(src) + off, n, cudaMemcpyDeviceToHost, cs));
    CMM_CUDA(cudaEventRecord(st.event(i), cs));
    inflight.push_back({off, n, i, s});
  }
  while (!inflight.empty()) drain();
}

}  // namespace cmm
