// Distance kernels for sm_100a: the reference's per-primitive distance_to_surface over a batch
// of (primitive, point) pairs, and the scene-level nearest-surface query (distance_core.cuh
// holds the arithmetic and the traversal).  Compiled with --fmad=false like the traversal, so
// that every distance equals the oracle's bit for bit.
//
// One thread per point, grid-stride over the batch.  The per-primitive form reads 28 bytes of
// query and writes 8 (plus 24 for closest points) and gathers one primitive record; the scene
// form walks the triangle and sphere BVHs nearest child first with a thread-local stack.
#include <cmath>

#include "alloc.h"
#include "bucket_sort.cuh"
#include "distance.h"
#include "distance_core.cuh"

namespace bzr {
namespace {

constexpr int kDistanceThreads = 256;
constexpr uint32_t kNearestStack = 64;

// One kind per instantiation, so that each kind's pass carries only its own code (registers,
// occupancy): spheres and planes are a gather and a few flops per query.
template <int KIND>
__global__ void __launch_bounds__(kDistanceThreads)
    distance_kernel(const SceneView S, const DistanceIO io) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < io.n; i += stride) {
    const D3 p = d3(io.points[3 * i], io.points[3 * i + 1], io.points[3 * i + 2]);
    D3 c;
    bool bad = false;
    io.distance[i] = distance_query(S, KIND, io.ids[i], p, &c, &bad);
    if (io.closest) {
      io.closest[3 * i] = c.x;
      io.closest[3 * i + 1] = c.y;
      io.closest[3 * i + 2] = c.z;
    }
    if (bad && io.error_word) flag_error(io.error_word, kErrPrimIndex);
  }
}

// Cylinders: the ellipse search takes 0 to 100 Newton steps per point (a quarter of random
// points run all 100), so a warp of 32 fixed queries would idle most lanes while its slowest
// one iterates.  Here each warp owns a contiguous range of queries and refills idle lanes from
// it: every trip of the loop gives new queries to the idle lanes (their decisions before the
// search, cylinder_setup) and one search step to the lanes in a search, all four sectors in
// the same instructions.
__global__ void __launch_bounds__(kDistanceThreads, 4)
    cylinder_distance_kernel(const SceneView S, const DistanceIO io) {
  const KindView &K = S.k[kCylinders];
  const unsigned full = 0xFFFFFFFFu;
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const uint64_t warps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  const uint64_t per = (io.n + warps - 1) / warps;
  uint64_t cursor = warp * per;
  const uint64_t end = cursor + per < io.n ? cursor + per : io.n;
  bool busy = false;
  uint64_t i = 0;
  CylinderQuery q;
  for (;;) {
    const unsigned idle = __ballot_sync(full, !busy);
    if (idle && cursor < end) {
      if (!busy) {
        const uint64_t j = cursor + __popc(idle & ((1u << lane) - 1u));
        if (j < end) {
          i = j;
          const D3 p = d3(io.points[3 * i], io.points[3 * i + 1], io.points[3 * i + 2]);
          const uint32_t id = io.ids[i];
          if (id >= K.n_prims) {
            io.distance[i] = bitsd(0x7FF8000000000000LL);
            if (io.error_word) flag_error(io.error_word, kErrPrimIndex);
          } else {
            const double *P = K.payload + size_t(payload_doubles(kCylinders)) * ldg(K.pos_of + id);
            double r[15];
            for (int k = 0; k < 15; ++k) r[k] = ldg(P + k);
            q = cylinder_setup(d3(r[0], r[1], r[2]), r[3], r[4], r[5], r + 6, p);
            if (q.region == 0)
              io.distance[i] = q.result;
            else
              busy = true;
          }
        }
      }
      cursor += __popc(idle);
    }
    if (!__any_sync(full, busy)) {
      if (cursor >= end) break;
      continue;
    }
    if (busy && !cylinder_search_step(q)) {
      io.distance[i] = cylinder_finish(q, q.v);
      busy = false;
    }
  }
}

__global__ void __launch_bounds__(kDistanceThreads)
    nearest_kernel(const SceneView S, const DistanceIO io) {
  uint32_t stack_ref[kNearestStack];
  float stack_key[kNearestStack];
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < io.n; j += stride) {
    const uint64_t i = io.perm ? io.perm[j] : j;
    const D3 p = d3(io.points[3 * i], io.points[3 * i + 1], io.points[3 * i + 2]);
    const NearestState st = nearest_surface(S, p, stack_ref, stack_key, kNearestStack);
    io.distance[i] = st.best;
    if (io.prim) io.prim[i] = st.prim;
    if (io.geom) io.geom[i] = st.geom;
  }
}

// Morton code of a point quantised to 512 cells per axis inside [lo, lo + 512 / scale),
// shifted to the top of the key.
__global__ void point_key_kernel(const double *points, uint32_t n, float3 lo, float3 scale,
                                 uint32_t *keys, uint32_t *counts) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float l[3] = {lo.x, lo.y, lo.z}, sc[3] = {scale.x, scale.y, scale.z};
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
      float x = (float(points[3 * size_t(i) + a]) - l[a]) * sc[a];
      x = fminf(fmaxf(x, 0.0f), 511.0f);  // NaN maps to 0
      q[a] = uint32_t(x);
    }
    const uint32_t k = ((spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2])) << 5;
    keys[i] = k;
    atomicAdd(counts + (k >> (32 - kSortBits)), 1u);
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
  const int grid = grid_of(io.n, sms, 8);
  switch (kind) {
    case kMesh:
      distance_kernel<kMesh><<<grid, kDistanceThreads, 0, stream>>>(S, io);
      break;
    case kSpheres:
      distance_kernel<kSpheres><<<grid, kDistanceThreads, 0, stream>>>(S, io);
      break;
    case kPlanes:
      distance_kernel<kPlanes><<<grid, kDistanceThreads, 0, stream>>>(S, io);
      break;
    default:
      cylinder_distance_kernel<<<grid, kDistanceThreads, 0, stream>>>(S, io);
      break;
  }
  return cudaGetLastError();
}

cudaError_t launch_nearest(const SceneView &S, const DistanceIO &io, int sms, cudaMemPool_t pool,
                           cudaStream_t stream) {
  if (io.n == 0) return cudaSuccess;
  DistanceIO run = io;
  uint32_t *scratch = nullptr;
  cudaError_t e = cudaSuccess;
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  bool any = false;
  for (int k = 0; k < kNumKinds; ++k) {
    const KindView &K = S.k[k];
    if (!K.present || K.n_prims == 0) continue;
    for (int a = 0; a < 3; ++a) {
      const double l = K.root_box[2 * a], h = K.root_box[2 * a + 1];
      lo[a] = any ? fmin(lo[a], l) : l;
      hi[a] = any ? fmax(hi[a], h) : h;
    }
    any = true;
  }
  if (any && pool && io.n >= kNearestSortMin && io.n < 0xFFFFFFFFull) {
    const uint32_t n = uint32_t(io.n);
    const size_t nb = size_t(1) << kSortBits;
    e = bzr::pool_malloc(&scratch,
                                (2 * size_t(n) + nb) * sizeof(uint32_t), pool, stream);
    if (e != cudaSuccess) return e;
    uint32_t *keys = scratch, *perm = scratch + n, *counts = scratch + 2 * size_t(n);
    float3 flo, fsc;
    float *pl = &flo.x, *ps = &fsc.x;
    for (int a = 0; a < 3; ++a) {
      const double ext = hi[a] - lo[a];
      pl[a] = float(lo[a]);
      ps[a] = ext > 0 && std::isfinite(ext) ? float(512.0 / ext) : 0.0f;
    }
    e = cudaMemsetAsync(counts, 0, nb * sizeof(uint32_t), stream);
    if (e == cudaSuccess) {
      const int blocks = (sms > 0 ? sms : 148) * 8;
      point_key_kernel<<<blocks, 256, 0, stream>>>(io.points, n, flo, fsc, keys, counts);
      bucket_scan_kernel<<<1, 1024, 0, stream>>>(counts);
      bucket_scatter_kernel<<<blocks, 256, 0, stream>>>(n, keys, counts, perm);
      e = cudaGetLastError();
      run.perm = perm;
    }
  }
  if (e == cudaSuccess) {
    nearest_kernel<<<grid_of(io.n, sms, 8), kDistanceThreads, 0, stream>>>(S, run);
    e = cudaGetLastError();
  }
  if (scratch) cudaFreeAsync(scratch, stream);
  return e;
}

}  // namespace bzr
