// Static device scratch for cmm_dev_compressed_product_noalloc.
//
// One file-scope device array of kNoAllocScratchBytes per device, reserved
// when this translation unit's module loads (with lazy module loading: at
// the first use of the symbol).  Its address is looked up with
// cudaGetSymbolAddress once per device and cached; the allocation-free entry
// point carves every intermediate of the slab pipeline out of it.  A single
// array per device means calls that overlap in time (other streams, other
// host threads) race on it.
#include <mutex>

#include "cmm_internal.h"

namespace cmm {

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

void* noalloc_scratch() {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static void* base[kMaxDevices] = {};
  int dev = 0;
  CMM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw unsupported("device ordinal above 63");
  std::lock_guard<std::mutex> g(mu);
  if (!base[dev]) {
    void* p = nullptr;
    CMM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (reinterpret_cast<uintptr_t>(p) % 256 != 0) throw cuda_error("static scratch is not 256-byte aligned");
    base[dev] = p;
  }
  return base[dev];
}

}  // namespace cmm
