// bzr_intersectN_noalloc: the batched closest-hit query for callers that cannot allocate device
// memory while they trace.
//
// Some callers of this library run inside another program that owns the device: a renderer
// plugin traced from the host application's frame loop, or a service whose device memory is
// handed out once, up front, by its host.  For them a cudaMalloc or cudaFree during a query is
// not acceptable: it synchronises the whole device (stalling the host's frame) or fails because
// the memory budget is already spent.  bzr_intersectN allocates in two places per call -- a
// stream-ordered scratch for the closest distance carried between the per-kind passes when the
// caller asks for no distances, and one for the coherence sort's buffers and the list of rays a
// mixed-precision pass hands to its FP64 pass.  This entry point needs no allocation: its
// scratch (the per-pass work counters, that distance carry and that list) lives in one
// file-scope device array, kScratchBytes long, which every GPU that loads this library holds
// until the process exits; it does not sort.
//
// Limits and rules:
//  * at most kMaxRays rays per call (the distance carry and the list take 12 bytes per ray);
//    larger batches are rejected with BZR_EINVAL -- split them;
//  * every array must be device memory of the scene's device; the work is queued on `stream`;
//  * every call on a device shares the one array and it keeps the last call's contents: the call
//    clears the work counters it needs on `stream` before its kernels run, but two calls whose
//    GPU work overlaps (for example on two streams) race on the array and give wrong results --
//    order them on one stream or with events;
//  * the first call on each device looks up the array's device address (cudaGetSymbolAddress,
//    with that device current) and caches it; make that first call before any stream capture;
//  * a device reset (cudaDeviceReset) ends the context the cached address belongs to, as it
//    frees every scene of that device: do not use this entry point on a device after
//    resetting it in the same process.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/blazert_b200.h"
#include "capi_internal.h"
#include "trace.h"

namespace {

constexpr size_t kMaxRays = size_t(1) << 20;                  // 1,048,576 rays per call
constexpr size_t kCounterBytes = 256;  // launch_trace's counters
constexpr size_t kDeferOffset = kCounterBytes + 8 * kMaxRays;  // after the distance carry
constexpr size_t kScratchBytes = kDeferOffset + 4 * kMaxRays;  // 12 MiB + 256 B per device
static_assert(bzr::kTraceCounterWords * sizeof(uint32_t) <= kCounterBytes, "counter words");
constexpr int kMaxDevices = 64;

// The scratch of every call on this device.  In host code the name is only a stand-in for
// the symbol: its device address comes from cudaGetSymbolAddress (scratch_address below).
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// Device address of g_scratch on `device` (which must be current); looked up once per device.
cudaError_t scratch_address(int device, unsigned char **out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return e;
    g_addr[device] = p;
  }
  *out = static_cast<unsigned char *>(g_addr[device]);
  return cudaSuccess;
}

}  // namespace

extern "C" int bzr_intersectN_noalloc(const bzr_scene *scene, size_t n, const double *origins,
                                      const double *directions, const double *tmin,
                                      const double *tmax, double *hit_distance, double *uv,
                                      double *normal, uint32_t *prim_id, uint32_t *geom_id,
                                      uint8_t *hit, int mode, void *stream) {
  bzr::SceneHandles h;
  const int rc = bzr::scene_handles(scene, &h);
  if (rc != BZR_OK) return rc;
  if (mode != BZR_MODE_FP64 && mode != BZR_MODE_MIXED)
    return bzr::set_error(BZR_EINVAL, "bad mode");
  if (n == 0) return BZR_OK;
  if (n > kMaxRays)
    return bzr::set_error(BZR_EINVAL,
                          "bzr_intersectN_noalloc takes at most 1,048,576 rays per call");
  if (!origins || !directions) return bzr::set_error(BZR_EINVAL, "origins and directions are required");
  const void *ptrs[10] = {origins, directions, tmin,    tmax,    hit_distance,
                          uv,      normal,     prim_id, geom_id, hit};
  for (const void *p : ptrs)
    if (p && !bzr::is_device_pointer(p))
      return bzr::set_error(BZR_EINVAL, "bzr_intersectN_noalloc takes device arrays only");
  if (h.device < 0 || h.device >= kMaxDevices) return bzr::set_error(BZR_EINVAL, "device index");
  int cur = 0;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return bzr::set_error(BZR_ECUDA, cudaGetErrorString(e));
  if (cur != h.device && (e = cudaSetDevice(h.device)) != cudaSuccess)
    return bzr::set_error(BZR_ECUDA, cudaGetErrorString(e));
  unsigned char *scratch = nullptr;
  e = scratch_address(h.device, &scratch);
  if (e == cudaSuccess) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    bzr::RayIO io;
    io.n = static_cast<uint32_t>(n);
    io.org = origins;
    io.dir = directions;
    io.tmin = tmin;
    io.tmax = tmax;
    io.t = hit_distance ? hit_distance : reinterpret_cast<double *>(scratch + kCounterBytes);
    io.uv = uv;
    io.normal = normal;
    io.prim = prim_id;
    io.geom = geom_id;
    io.hit = hit;
    io.error_word = h.error_word;
    io.defer = reinterpret_cast<uint32_t *>(scratch + kDeferOffset);
    bzr::LaunchPlan plan = *h.plan;
    plan.sort.enabled = false;  // the sort would need per-call buffers
    // launch_trace clears the counters on `st` before the kernels run
    e = bzr::launch_trace(*h.view, io, mode, plan, st, reinterpret_cast<uint32_t *>(scratch));
  }
  if (cur != h.device) {
    const cudaError_t back = cudaSetDevice(cur);  // the caller's device, as it was
    if (e == cudaSuccess) e = back;
  }
  if (e != cudaSuccess) return bzr::set_error(BZR_ECUDA, cudaGetErrorString(e));
  return BZR_OK;
}
