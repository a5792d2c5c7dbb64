// Host interface of the traversal kernels (trace.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "layout.h"

namespace bzr {

constexpr int kTraceThreads = 128;

// Device pointers of one batch.  tmin / tmax may be null (0 and DBL_MAX); each output may be
// null.  work_counter must be zero when the kernel starts; error_word collects kErr* bits.
struct RayIO {
  const double *org = nullptr;
  const double *dir = nullptr;
  const double *tmin = nullptr;
  const double *tmax = nullptr;
  double *t = nullptr;
  double *uv = nullptr;
  double *normal = nullptr;
  uint32_t *prim = nullptr;
  uint32_t *geom = nullptr;
  uint8_t *hit = nullptr;
  uint32_t n = 0;
  uint32_t *work_counter = nullptr;
  uint32_t *error_word = nullptr;
};

size_t trace_smem_bytes(uint32_t stack_cap, int threads);
// Persistent grid size for the current device: SMs x resident blocks per SM.
cudaError_t trace_grid(uint32_t stack_cap, int *blocks);
// totals (device, 8 x uint64, or null): when given, the counting kernel also adds per kind the
// box tests (totals[0..3]) and primitive tests (totals[4..7]) of every ray.
cudaError_t launch_trace(const SceneView &S, const RayIO &io, int mode, int blocks,
                         cudaStream_t stream, unsigned long long *totals = nullptr);

}  // namespace bzr
