// Distance kernels for sm_100a: the reference's per-primitive distance_to_surface over a batch
// of (primitive, point) pairs, and the scene-level nearest-surface query (distance_core.cuh
// holds the arithmetic and the traversal).  Compiled with --fmad=false like the traversal, so
// that every distance equals the oracle's bit for bit.
//
// One thread per point, grid-stride over the batch.  The per-primitive form reads 28 bytes of
// query and writes 8 (plus 24 for closest points) and gathers one primitive record; the scene
// form walks the triangle and sphere BVHs nearest child first with a thread-local stack.
#include "distance.h"
#include "distance_core.cuh"

namespace bzr {
namespace {

constexpr int kDistanceThreads = 256;
constexpr uint32_t kNearestStack = 64;

__global__ void __launch_bounds__(kDistanceThreads)
    distance_kernel(const SceneView S, const int kind, const DistanceIO io) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < io.n; i += stride) {
    const D3 p = d3(io.points[3 * i], io.points[3 * i + 1], io.points[3 * i + 2]);
    D3 c;
    bool bad = false;
    io.distance[i] = distance_query(S, kind, io.ids[i], p, &c, &bad);
    if (io.closest) {
      io.closest[3 * i] = c.x;
      io.closest[3 * i + 1] = c.y;
      io.closest[3 * i + 2] = c.z;
    }
    if (bad && io.error_word) flag_error(io.error_word, kErrPrimIndex);
  }
}

__global__ void __launch_bounds__(kDistanceThreads)
    nearest_kernel(const SceneView S, const DistanceIO io) {
  uint32_t stack_ref[kNearestStack];
  double stack_key[kNearestStack];
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < io.n; i += stride) {
    const D3 p = d3(io.points[3 * i], io.points[3 * i + 1], io.points[3 * i + 2]);
    const NearestState st = nearest_surface(S, p, stack_ref, stack_key, kNearestStack);
    io.distance[i] = st.best;
    if (io.prim) io.prim[i] = st.prim;
    if (io.geom) io.geom[i] = st.geom;
  }
}

int grid_of(uint64_t n, int sms, int per_sm) {
  const uint64_t want = (n + kDistanceThreads - 1) / kDistanceThreads;
  const uint64_t cap = uint64_t(sms > 0 ? sms : 148) * per_sm;
  return int(want < cap ? want : cap);
}

}  // namespace

cudaError_t launch_distance(const SceneView &S, int kind, const DistanceIO &io, int sms,
                            cudaStream_t stream) {
  if (io.n == 0) return cudaSuccess;
  distance_kernel<<<grid_of(io.n, sms, 8), kDistanceThreads, 0, stream>>>(S, kind, io);
  return cudaGetLastError();
}

cudaError_t launch_nearest(const SceneView &S, const DistanceIO &io, int sms,
                           cudaStream_t stream) {
  if (io.n == 0) return cudaSuccess;
  nearest_kernel<<<grid_of(io.n, sms, 8), kDistanceThreads, 0, stream>>>(S, io);
  return cudaGetLastError();
}

}  // namespace bzr
