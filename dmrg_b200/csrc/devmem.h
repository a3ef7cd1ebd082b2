// Stream-ordered device allocations from the device's default memory pool: a
// free is queued behind the work already on the stream instead of
// synchronising the whole device, so contexts on different streams (and host
// threads) do not wait for each other's kernels.  Internal header.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>

namespace dmrgx {

template <class T>
inline cudaError_t dalloc(T** p, size_t count, cudaStream_t s) {
  return cudaMallocAsync(reinterpret_cast<void**>(p), sizeof(T) * std::max<size_t>(1, count), s);
}
inline void dfree(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

// Keep memory freed into the pool cached by the process (the pool otherwise
// returns it to the driver at every synchronisation).  Process-local setting.
inline void keep_pool(int device) {
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
}

}  // namespace dmrgx
