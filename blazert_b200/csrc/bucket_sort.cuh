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

// In-place exclusive scan of the 2^kSortBits counts; one block of 1024 threads (32 warps).
// Each warp scans its contiguous 2,048 counts in coalesced rounds of 32 (shuffle scan, running
// carry), the 32 warp totals are scanned by one warp, and a second coalesced pass adds each
// warp's offset.
__global__ void __launch_bounds__(1024) bucket_scan_kernel(uint32_t *counts) {
  constexpr int kPerWarp = (1 << kSortBits) / 32;
  constexpr unsigned kFull = 0xFFFFFFFFu;
  __shared__ uint32_t warp_offset[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *c = counts + warp * kPerWarp;
  uint32_t carry = 0;
  for (int r = 0; r < kPerWarp; r += 32) {
    const uint32_t v = c[r + lane];
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    c[r + lane] = carry + x - v;
    carry += __shfl_sync(kFull, x, 31);
  }
  if (lane == 0) warp_offset[warp] = carry;
  __syncthreads();
  if (warp == 0) {
    const uint32_t t = warp_offset[lane];
    uint32_t x = t;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    warp_offset[lane] = x - t;
  }
  __syncthreads();
  const uint32_t off = warp_offset[warp];
  for (int r = 0; r < kPerWarp; r += 32) c[r + lane] += off;
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
