// Device counting sort on the top kSortBits bits of 32-bit keys, shared by the ray coherence
// sort (trace.cu) and the point sort of the nearest-surface query (distance.cu).  Three
// launches: the caller's histogram kernel (keys and bucket counts), bucket_scan_kernel
// (exclusive scan of the counts in place), bucket_scatter_kernel (perm[position] = index).
// Within a bucket the order is that of the atomics; only the processing order depends on it.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace bzr {

constexpr int kSortBits = 16;

__device__ __forceinline__ uint32_t spread3(uint32_t v) {  // 9 bits -> every third bit
  v &= 0x1FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

namespace {

// In-place exclusive scan of 2^kSortBits counts; one block of 1024 threads.
__global__ void __launch_bounds__(1024) bucket_scan_kernel(uint32_t *counts) {
  constexpr int kPer = (1 << kSortBits) / 1024;
  __shared__ uint32_t part[1024];
  uint32_t *c = counts + threadIdx.x * kPer;
  uint32_t sum = 0;
  for (int j = 0; j < kPer; ++j) sum += c[j];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {  // Hillis-Steele inclusive scan
    const uint32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = part[threadIdx.x] - sum;
  for (int j = 0; j < kPer; ++j) {
    const uint32_t v = c[j];
    c[j] = run;
    run += v;
  }
}

__global__ void bucket_scatter_kernel(uint32_t n, const uint32_t *keys, uint32_t *offsets,
                                      uint32_t *perm) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t pos = atomicAdd(offsets + (keys[i] >> (32 - kSortBits)), 1u);
    if (pos < n) perm[pos] = i;
  }
}

}  // namespace
}  // namespace bzr
