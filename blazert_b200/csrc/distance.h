// Host interface of the distance kernels (distance.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "layout.h"

namespace bzr {

// Device pointers of one distance batch of n points.  Per-primitive form: ids[i] names the
// primitive of the kind, closest (triangles, may be null) receives n x 3 closest points.
// Scene form: prim / geom (may be null) receive the nearest primitive's ids.
struct DistanceIO {
  uint64_t n = 0;
  const uint32_t *ids = nullptr;
  const double *points = nullptr;  // n x 3
  double *distance = nullptr;      // n
  double *closest = nullptr;       // n x 3
  uint32_t *prim = nullptr;
  uint32_t *geom = nullptr;
  uint32_t *error_word = nullptr;  // kErrPrimIndex for an id outside the kind
  const uint32_t *perm = nullptr;  // optional processing order of the scene form
};

cudaError_t launch_distance(const SceneView &S, int kind, const DistanceIO &io, int sms,
                            cudaStream_t stream);
// Batches of at least kNearestSortMin points are processed in the order of a Morton code of
// the point inside the scene's box (a device counting sort with scratch from `pool`), so that
// the lanes of a warp search neighbouring regions of the BVHs; results go to each point's
// own index.
constexpr uint64_t kNearestSortMin = 1u << 16;
cudaError_t launch_nearest(const SceneView &S, const DistanceIO &io, int sms, cudaMemPool_t pool,
                           cudaStream_t stream);

}  // namespace bzr
