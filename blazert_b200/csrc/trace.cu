// Closest-hit traversal kernels for sm_100a.
//
// One thread per ray, persistent warps that fetch 32 rays at a time from a global counter.
// Per ray the per-kind BVHs are traversed in the reference's fixed order (triangles, spheres,
// planes, cylinders; blazert/scene.h:161-210) and merged with its strict "<".
//
// Exactness.  The kernels reproduce the reference's visit order and arithmetic bit for bit:
//  * compiled with --fmad=false; every expression keeps the reference's evaluation order;
//  * the reference pushes both children of a node and tests a node's box when it is POPPED,
//    against the hit distance current at that moment (blazert/bvh/accel.h:89-113).  Here the
//    parent tests both children at once.  For each child the slab test splits into a part that
//    does not depend on the hit distance h (entry mn <= exit E, with E evaluated as if
//    h = +inf) and the comparison mn <= h, which is deferred to pop time (the stack stores mn
//    as the key).  When an exit distance is NaN (0 * inf on a slab plane) the reference's
//    std::min chain drops h entirely; the key is then -inf so that the pop test always passes.
//    The result is the reference's sequence of accepted nodes, including nodes re-accepted
//    after a cylinder hit moved h outward (cylinders do not test against h,
//    blazert/primitives/cylinder.h:181-495).
//  * the slab test keeps the reference's far-plane factor l1 = 1 + 4 eps and its std::max /
//    std::min argument order (blazert/bvh/intersect.h:33-51).
#include <cuda_runtime.h>

#include <cstdint>

#include "layout.h"
#include "trace.h"
#include "trace_core.cuh"

namespace bzr {
namespace {

// COUNT = true: also sums the work counters of all rays into totals[8] (box tests per kind,
// then primitive tests per kind); used to derive the algorithmic bytes of a workload.
template <bool COUNT>
__global__ void __launch_bounds__(kTraceThreads)
    trace_fp64_kernel(SceneView S, RayIO io, unsigned long long *totals) {
  extern __shared__ __align__(16) unsigned char smem[];
  Stack sk;
  sk.stride = blockDim.x;
  sk.cap = S.stack_cap;
  sk.key = reinterpret_cast<double *>(smem);
  sk.ref = reinterpret_cast<uint32_t *>(sk.key + size_t(sk.cap) * sk.stride);
  const unsigned lane = threadIdx.x & 31u;
  Counts cnt = {};
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(io.work_counter, 32u);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (base >= io.n) break;
    const uint64_t i = uint64_t(base) + lane;
    if (i >= io.n) continue;
    const Ray r = make_ray(io.org + 3 * i, io.dir + 3 * i, io.tmin ? io.tmin[i] : 0.0,
                           io.tmax ? io.tmax[i] : kDblMax);
    Best best;
    trace_ray<COUNT>(S, r, sk, threadIdx.x, io.error_word, best, &cnt);
    if (io.t) io.t[i] = best.t;
    if (io.uv) {
      io.uv[2 * i] = best.u;
      io.uv[2 * i + 1] = best.v;
    }
    if (io.normal) {
      io.normal[3 * i] = best.n.x;
      io.normal[3 * i + 1] = best.n.y;
      io.normal[3 * i + 2] = best.n.z;
    }
    if (io.prim) io.prim[i] = best.prim;
    if (io.geom) io.geom[i] = best.geom;
    if (io.hit) io.hit[i] = best.hit ? 1 : 0;
  }
  if (COUNT) {
    for (int k = 0; k < kNumKinds; ++k) {
      unsigned long long b = cnt.box[k], p = cnt.prim[k];
      for (int off = 16; off > 0; off >>= 1) {
        b += __shfl_down_sync(0xFFFFFFFFu, b, off);
        p += __shfl_down_sync(0xFFFFFFFFu, p, off);
      }
      if (lane == 0) {
        atomicAdd(totals + k, b);
        atomicAdd(totals + kNumKinds + k, p);
      }
    }
  }
}

}  // namespace

size_t trace_smem_bytes(uint32_t stack_cap, int threads) {
  return size_t(stack_cap) * threads * (sizeof(double) + sizeof(uint32_t));
}

cudaError_t trace_grid(uint32_t stack_cap, int *blocks) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const size_t smem = trace_smem_bytes(stack_cap, kTraceThreads);
  e = cudaFuncSetAttribute(trace_fp64_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(smem));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(trace_fp64_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(smem));
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_fp64_kernel<false>,
                                                    kTraceThreads, smem);
  if (e != cudaSuccess) return e;
  *blocks = sms * (per_sm > 0 ? per_sm : 1);
  return cudaSuccess;
}

cudaError_t launch_trace(const SceneView &S, const RayIO &io, int mode, int blocks,
                         cudaStream_t stream, unsigned long long *totals) {
  (void)mode;
  const size_t smem = trace_smem_bytes(S.stack_cap, kTraceThreads);
  if (totals)
    trace_fp64_kernel<true><<<blocks, kTraceThreads, smem, stream>>>(S, io, totals);
  else
    trace_fp64_kernel<false><<<blocks, kTraceThreads, smem, stream>>>(S, io, nullptr);
  return cudaGetLastError();
}

}  // namespace bzr
