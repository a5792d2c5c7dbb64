// Device and pinned-host allocations of the library go through these wrappers, so that a test
// can make the k-th of them fail (bzr_debug_fail_allocation) and check that every entry point
// then reports BZR_ENOMEM and releases what it had allocated.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

namespace bzr {

// True when the armed countdown of bzr_debug_fail_allocation reaches this allocation (capi.cpp).
bool injected_allocation_failure();

template <class T>
cudaError_t dev_malloc(T **p, size_t bytes) {
  if (injected_allocation_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(reinterpret_cast<void **>(p), bytes);
}

template <class T>
cudaError_t host_malloc(T **p, size_t bytes) {
  if (injected_allocation_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocHost(reinterpret_cast<void **>(p), bytes);
}

template <class T>
cudaError_t pool_malloc(T **p, size_t bytes, cudaMemPool_t pool, cudaStream_t stream) {
  if (injected_allocation_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocFromPoolAsync(reinterpret_cast<void **>(p), bytes, pool, stream);
}

}  // namespace bzr
