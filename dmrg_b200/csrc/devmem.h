// Stream-ordered device allocations from a memory pool private to the library:
// a free is queued behind the work already on the stream instead of
// synchronising the whole device, so contexts on different streams (and host
// threads) do not wait for each other's kernels.  Internal header.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <mutex>

namespace dmrgx {

// The library's own pool on `device`, created on first use: freed memory stays
// cached in it (release threshold: no limit) instead of going back to the
// driver at every synchronisation.  The device's default pool, which the host
// application may allocate from, is left untouched.  Null if the pool cannot be
// created.
inline cudaMemPool_t library_pool(int device) {
  constexpr int kMaxDev = 64;
  static std::mutex mu;
  static cudaMemPool_t pools[kMaxDev] = {};
  if (device < 0 || device >= kMaxDev) return nullptr;
  std::lock_guard<std::mutex> g(mu);
  if (!pools[device]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    pools[device] = pool;
  }
  return pools[device];
}

// Stream-ordered allocation from the library pool of the stream's device.
template <class T>
inline cudaError_t dalloc(T** p, size_t count, cudaStream_t s) {
  int dev = 0;
  cudaError_t e = cudaStreamGetDevice(s, &dev);
  if (e != cudaSuccess) return e;
  cudaMemPool_t pool = library_pool(dev);
  if (!pool) return cudaErrorMemoryAllocation;
  return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p),
                                 sizeof(T) * std::max<size_t>(1, count), pool, s);
}
inline void dfree(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

}  // namespace dmrgx
