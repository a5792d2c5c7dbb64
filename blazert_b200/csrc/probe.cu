// Read-bandwidth probe for the roofline's cache ceiling (measurement only; not part of the
// query path).
//
// The traversal kernels read nodes and primitives that mostly come from L1 and L2, not DRAM,
// so their byte ceiling is the L2's read bandwidth, which nothing in the CUDA toolkit states.
// bzr_probe_read_gbs measures it: a buffer of `bytes` is read `reps` times by a grid of
// (SMs x 8) blocks of 256 threads with 16-byte loads.  With l1_bypass set the loads are
// ld.global.cg (cached in L2 only), so a buffer that fits in L2 measures L2 -> SM bandwidth;
// without it they are ordinary loads (L1 and L2).  The first pass is untimed (it brings the
// buffer into the caches); the timed passes are bracketed by CUDA events on one stream.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace {

template <bool CG>
__global__ void __launch_bounds__(256) read_kernel(const uint4 *__restrict__ p, size_t n16,
                                                   int reps, unsigned *sink) {
  uint32_t acc = 0;
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (int r = 0; r < reps; ++r) {
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n16; i += 4 * stride) {
      uint4 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = CG ? __ldcg(p + i + u * stride) : p[i + u * stride];
#pragma unroll
      for (int u = 0; u < 4; ++u) acc ^= v[u].x ^ v[u].y ^ v[u].z ^ v[u].w;
    }
    for (; i < n16; i += stride) {
      const uint4 v = CG ? __ldcg(p + i) : p[i];
      acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
  }
  if (acc == 0x9E3779B9u) *sink = acc;  // keeps the loads; the buffer holds no such pattern
}

}  // namespace

// Measured read bandwidth in GB/s (1e9 bytes per second) into *gbs; 0 on success, else the
// CUDA error code.  Allocates and frees its own buffer on the current device.
extern "C" int bzr_probe_read_gbs(size_t bytes, int reps, int l1_bypass, double *gbs) {
  if (!gbs || bytes < 16 || reps < 1) return int(cudaErrorInvalidValue);
  *gbs = 0.0;
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return int(e);
  const size_t n16 = bytes / 16;
  void *buf = nullptr;
  unsigned *sink = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  if ((e = cudaMalloc(&buf, n16 * 16 + 256)) != cudaSuccess) return int(e);
  sink = reinterpret_cast<unsigned *>(static_cast<char *>(buf) + n16 * 16);
  float ms = 0.0f;
  e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMemsetAsync(buf, 0x5A, n16 * 16, st);
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  if (e == cudaSuccess) {
    const uint4 *p = static_cast<const uint4 *>(buf);
    const int grid = sms * 8;
    if (l1_bypass) read_kernel<true><<<grid, 256, 0, st>>>(p, n16, 1, sink);
    else read_kernel<false><<<grid, 256, 0, st>>>(p, n16, 1, sink);
    cudaEventRecord(a, st);
    if (l1_bypass) read_kernel<true><<<grid, 256, 0, st>>>(p, n16, reps, sink);
    else read_kernel<false><<<grid, 256, 0, st>>>(p, n16, reps, sink);
    cudaEventRecord(b, st);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventSynchronize(b);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  if (e == cudaSuccess && ms > 0.0f) *gbs = double(n16) * 16.0 * reps / (double(ms) * 1e-3) / 1e9;
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (st) cudaStreamDestroy(st);
  cudaFree(buf);
  return int(e);
}
