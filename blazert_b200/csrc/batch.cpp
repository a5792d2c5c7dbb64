// C-ABI of the batching form: many committed scenes, each with its own batch of rays, traced by
// one persistent kernel per primitive kind, the launch sequence captured in a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "alloc.h"
#include "../../include/blazert_b200.h"
#include "capi_internal.h"
#include "trace.h"

struct bzr_batch {
  int device = -1;
  std::vector<const bzr_scene *> scenes;
  std::vector<bzr::SceneView> views;
  std::vector<int8_t> first_kind, last_kind;
  bzr::BatchPlan plan;
  // device memory: views, first/last kinds, per-scene rays and counters, chunk table
  bzr::SceneView *d_views = nullptr;
  int8_t *d_first = nullptr, *d_last = nullptr;
  uint32_t *d_rays = nullptr, *d_left = nullptr, *d_words = nullptr;  // words: 4 counters, error
  bzr::BatchChunk *d_chunks = nullptr;
  size_t chunk_cap = 0;
  // coherence sort (bzr_batch_tune BZR_TUNE_SORT): per-scene quantisation boxes, and the
  // keys, permutation and bucket counts (grown with the batch)
  bzr::RaySort *d_sort = nullptr;
  uint32_t *d_sort_words = nullptr;
  size_t sort_cap = 0;  // rays the sort scratch holds
  cudaStream_t capture = nullptr;
  // graph of the last argument set
  cudaGraphExec_t exec = nullptr;
  std::vector<uint64_t> key;
  std::mutex mu;

  ~bzr_batch() {
    if (device < 0) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    if (exec) cudaGraphExecDestroy(exec);
    if (capture) cudaStreamDestroy(capture);
    cudaFree(d_views);
    cudaFree(d_first);
    cudaFree(d_last);
    cudaFree(d_rays);
    cudaFree(d_left);
    cudaFree(d_words);
    cudaFree(d_chunks);
    cudaFree(d_sort);
    cudaFree(d_sort_words);
    cudaSetDevice(cur);
  }
};

namespace {
int fail(int code, const char *msg) { return bzr::set_error(code, msg); }
int cuda_fail(cudaError_t e) {
  return bzr::set_error(e == cudaErrorMemoryAllocation ? BZR_ENOMEM : BZR_ECUDA,
                        cudaGetErrorString(e));
}
}  // namespace

extern "C" {

int bzr_batch_create(bzr_batch **out, const bzr_scene *const *scenes, size_t n_scenes) {
  if (!out || !scenes || n_scenes == 0 || n_scenes > (1u << 24))
    return fail(BZR_EINVAL, "bad batch arguments");
  *out = nullptr;
  auto *b = new (std::nothrow) bzr_batch();
  if (!b) return fail(BZR_ENOMEM, "batch allocation failed");
  uint32_t cap = 8;
  for (size_t s = 0; s < n_scenes; ++s) {
    bzr::SceneHandles h;
    const int rc = bzr::scene_handles(scenes[s], &h);
    if (rc != BZR_OK) {
      delete b;
      return rc;
    }
    if (b->device >= 0 && h.device != b->device) {
      delete b;
      return fail(BZR_EINVAL, "all scenes of a batch must be on one device");
    }
    b->device = h.device;
    b->scenes.push_back(scenes[s]);
    b->views.push_back(*h.view);
    cap = std::max(cap, h.view->stack_cap);
    int8_t first = -1, last = -1;
    for (int k = 0; k < bzr::kNumKinds; ++k)
      if (h.view->k[k].present && h.view->k[k].n_prims) {
        if (first < 0) first = int8_t(k);
        last = int8_t(k);
        b->plan.kinds_present |= 1 << k;
      }
    b->first_kind.push_back(first);
    b->last_kind.push_back(last);
  }
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  cudaError_t e = bzr::batch_prepare(cap, &b->plan);
  const size_t n = n_scenes;
  if (e == cudaSuccess) e = bzr::dev_malloc(&b->d_views, n * sizeof(bzr::SceneView));
  if (e == cudaSuccess) e = bzr::dev_malloc(&b->d_first, n);
  if (e == cudaSuccess) e = bzr::dev_malloc(&b->d_last, n);
  if (e == cudaSuccess) e = bzr::dev_malloc(&b->d_rays, n * sizeof(uint32_t));
  if (e == cudaSuccess) e = bzr::dev_malloc(&b->d_left, n * sizeof(uint32_t));
  if (e == cudaSuccess) e = bzr::dev_malloc(&b->d_words, 8 * sizeof(uint32_t));
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_views, b->views.data(), n * sizeof(bzr::SceneView), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_first, b->first_kind.data(), n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_last, b->last_kind.data(), n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->d_words, 0, 8 * sizeof(uint32_t));
  if (e == cudaSuccess) {
    // per scene the box of its root boxes, as the single-scene coherence sort quantises origins
    std::vector<bzr::RaySort> sorts(n);
    for (size_t s = 0; s < n; ++s) {
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      for (int k = 0; k < bzr::kNumKinds; ++k) {
        const bzr::KindView &kv = b->views[s].k[k];
        if (!kv.present || !kv.n_prims) continue;
        for (int a = 0; a < 3; ++a) {
          lo[a] = std::min(lo[a], kv.root_box[2 * a]);
          hi[a] = std::max(hi[a], kv.root_box[2 * a + 1]);
        }
      }
      for (int a = 0; a < 3; ++a) {
        const double ext = hi[a] - lo[a];
        const bool finite = ext > 0.0 && ext < 1e300;
        sorts[s].lo[a] = finite ? float(lo[a]) : 0.0f;
        sorts[s].scale[a] = finite ? float(512.0 / ext) : 0.0f;
      }
      sorts[s].enabled = true;
    }
    e = bzr::dev_malloc(&b->d_sort, n * sizeof(bzr::RaySort));
    if (e == cudaSuccess)
      e = cudaMemcpy(b->d_sort, sorts.data(), n * sizeof(bzr::RaySort), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking);
  cudaSetDevice(cur);
  if (e != cudaSuccess) {
    delete b;
    return cuda_fail(e);
  }
  *out = b;
  return BZR_OK;
}

int bzr_batch_destroy(bzr_batch *b) {
  delete b;
  return BZR_OK;
}

int bzr_batch_intersect(bzr_batch *b, const uint64_t *ray_offsets, const double *origins,
                        const double *directions, const double *tmin, const double *tmax,
                        double *hit_distance, double *uv, double *normal, uint32_t *prim_id,
                        uint32_t *geom_id, uint8_t *hit, uint64_t *scene_done_ns, int mode,
                        void *stream) {
  if (!b || !ray_offsets || !origins || !directions || !hit_distance)
    return fail(BZR_EINVAL, "batch: offsets, origins, directions and hit_distance are required");
  if (mode != BZR_MODE_FP64 && mode != BZR_MODE_MIXED) return fail(BZR_EINVAL, "bad mode");
  const size_t ns = b->scenes.size();
  if (ray_offsets[0] != 0) return fail(BZR_EINVAL, "ray_offsets[0] must be 0");
  for (size_t s = 0; s < ns; ++s)
    if (ray_offsets[s + 1] < ray_offsets[s]) return fail(BZR_EINVAL, "ray_offsets decrease");
  const uint64_t total = ray_offsets[ns];
  if (total > 0x7FFFFF00ull) return fail(BZR_EINVAL, "batch too large (at most 2^31 rays)");
  const void *ptrs[] = {origins, directions, tmin, tmax, hit_distance, uv, normal, prim_id,
                        geom_id, hit, scene_done_ns};
  for (const void *p : ptrs)
    if (p && !bzr::is_device_pointer(p)) return fail(BZR_EINVAL, "batch arrays must be device memory");
  std::lock_guard<std::mutex> lock(b->mu);
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // graph key: everything the captured launches depend on
  std::vector<uint64_t> key(ray_offsets, ray_offsets + ns + 1);
  for (const void *p : ptrs) key.push_back(reinterpret_cast<uint64_t>(p));
  key.push_back(uint64_t(mode));
  cudaError_t e = cudaSuccess;
  if (!b->exec || key != b->key) {
    // chunk table and per-scene ray counts for these offsets
    std::vector<bzr::BatchChunk> chunks;
    std::vector<uint32_t> rays(ns);
    for (size_t s = 0; s < ns; ++s) {
      rays[s] = uint32_t(ray_offsets[s + 1] - ray_offsets[s]);
      // nothing to trace: filled with defaults below (a sorted batch still needs its chunks
      // to give its rays sort keys; the kernels skip scenes without the kind they trace)
      if (b->first_kind[s] < 0 && !b->plan.sort) continue;
      for (uint64_t a = ray_offsets[s]; a < ray_offsets[s + 1]; a += bzr::kBatchChunk)
        chunks.push_back({uint32_t(s), uint32_t(a),
                          uint32_t(std::min<uint64_t>(a + bzr::kBatchChunk, ray_offsets[s + 1]))});
    }
    if (chunks.size() > b->chunk_cap) {
      cudaFree(b->d_chunks);
      b->d_chunks = nullptr;
      b->chunk_cap = 0;
      e = bzr::dev_malloc(&b->d_chunks, std::max<size_t>(1, chunks.size()) * sizeof(bzr::BatchChunk));
      if (e != cudaSuccess) {
        cudaSetDevice(cur);
        return fail(BZR_ENOMEM, "chunk table allocation failed");
      }
      b->chunk_cap = chunks.size();
    }
    cudaStreamSynchronize(st);  // the previous graph may still read the tables
    if (!chunks.empty())
      e = cudaMemcpy(b->d_chunks, chunks.data(), chunks.size() * sizeof(bzr::BatchChunk),
                     cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(b->d_rays, rays.data(), ns * sizeof(uint32_t), cudaMemcpyHostToDevice);
    bzr::BatchSortScratch scratch;
    if (e == cudaSuccess && b->plan.sort) {
      if (total > b->sort_cap) {
        cudaFree(b->d_sort_words);
        b->d_sort_words = nullptr;
        b->sort_cap = 0;
        e = bzr::dev_malloc(&b->d_sort_words,
                            (2 * size_t(total) + bzr::kSortBuckets) * sizeof(uint32_t));
        if (e != cudaSuccess) {
          cudaSetDevice(cur);
          return fail(BZR_ENOMEM, "sort scratch allocation failed");
        }
        b->sort_cap = total;
      }
      scratch.keys = b->d_sort_words;
      scratch.perm = b->d_sort_words + total;
      scratch.counts = b->d_sort_words + 2 * total;
    }
    bzr::BatchView B;
    B.views = b->d_views;
    B.scene_sort = b->d_sort;
    for (B.scene_bits = 1; (size_t(1) << B.scene_bits) < ns; ++B.scene_bits) {
    }
    B.chunks = b->d_chunks;
    B.n_chunks = uint32_t(chunks.size());
    B.n_scenes = uint32_t(ns);
    B.first_kind = b->d_first;
    B.last_kind = b->d_last;
    B.scene_rays = b->d_rays;
    B.scene_left = b->d_left;
    B.scene_done_ns = reinterpret_cast<unsigned long long *>(scene_done_ns);
    B.start_ns = scene_done_ns ? reinterpret_cast<unsigned long long *>(scene_done_ns + ns) : nullptr;
    bzr::RayIO io;
    io.n = uint32_t(total);
    io.org = origins;
    io.dir = directions;
    io.tmin = tmin;
    io.tmax = tmax;
    io.t = hit_distance;
    io.uv = uv;
    io.normal = normal;
    io.prim = prim_id;
    io.geom = geom_id;
    io.hit = hit;
    io.error_word = b->d_words + bzr::kNumKinds;
    cudaGraph_t graph = nullptr;
    if (e == cudaSuccess) e = cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      cudaError_t le = bzr::launch_batch(B, io, mode, b->plan, b->capture, b->d_words, scratch);
      for (size_t s = 0; le == cudaSuccess && s < ns; ++s) {
        if (b->first_kind[s] >= 0 || ray_offsets[s + 1] == ray_offsets[s]) continue;
        bzr::RayIO sub = io;  // a scene with nothing to trace gets the RayHit defaults
        const uint64_t a = ray_offsets[s];
        sub.n = uint32_t(ray_offsets[s + 1] - a);
        sub.t = io.t + a;
        sub.uv = io.uv ? io.uv + 2 * a : nullptr;
        sub.normal = io.normal ? io.normal + 3 * a : nullptr;
        sub.prim = io.prim ? io.prim + a : nullptr;
        sub.geom = io.geom ? io.geom + a : nullptr;
        sub.hit = io.hit ? io.hit + a : nullptr;
        le = bzr::launch_defaults(sub, b->plan.sms, b->capture);
      }
      e = cudaStreamEndCapture(b->capture, &graph);
      if (e == cudaSuccess && le != cudaSuccess) e = le;
    }
    if (b->exec) {
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    b->key = e == cudaSuccess ? key : std::vector<uint64_t>();
  }
  if (e == cudaSuccess) e = cudaGraphLaunch(b->exec, st);
  cudaSetDevice(cur);
  return e == cudaSuccess ? BZR_OK : cuda_fail(e);
}

int bzr_batch_tune(bzr_batch *b, int option, int64_t value) {
  if (!b) return fail(BZR_EINVAL, "batch is null");
  std::lock_guard<std::mutex> lock(b->mu);
  bzr::BatchPlan p = b->plan;
  if (option == BZR_TUNE_BLOCK) {
    if (value != 64 && value != 128 && value != 256)
      return fail(BZR_EINVAL, "threads per block must be 64, 128 or 256");
    p.threads = static_cast<int>(value);
  } else if (option == BZR_TUNE_STACK) {
    if (value != 0 && value != 1) return fail(BZR_EINVAL, "stack storage must be 0 or 1");
    p.shared_stack = value == 1;
  } else if (option == BZR_TUNE_STACK_DEPTH) {
    if (value != 32 && value != 64)
      return fail(BZR_EINVAL, "the thread-local stack holds 32 or 64 entries");
    if (value == 32 && p.stack_cap > 32)
      return fail(BZR_EINVAL, "a scene of the batch needs more than 32 stack entries");
    p.local_stack = static_cast<uint32_t>(value);
  } else if (option == BZR_TUNE_SORT) {
    if (value != 0 && value != 1) return fail(BZR_EINVAL, "sort must be 0 or 1");
    if (value == 1 && b->scenes.size() > bzr::kBatchSortMaxScenes)
      return fail(BZR_EINVAL, "the coherence sort takes batches of at most 4,096 scenes");
    p.sort = value == 1;
  } else if (option == BZR_TUNE_NODE_WIDTH) {
    if (value != 2 && value != 8) return fail(BZR_EINVAL, "node width must be 2 or 8");
    p.node_width = static_cast<uint32_t>(value);
  } else {
    return fail(BZR_EINVAL, "unknown tuning option for a batch");
  }
  if ((p.shared_stack || p.stack_cap > bzr::kLocalStack) &&
      bzr::trace_smem_bytes(p.stack_cap, p.threads) > 227 * 1024)
    return fail(BZR_EINVAL, "the traversal stack does not fit shared memory at this block size");
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  cudaError_t e = bzr::batch_prepare(p.stack_cap, &p);
  if (e == cudaSuccess && b->exec) {  // the cached graph holds the old launch shape
    e = cudaStreamSynchronize(b->capture);
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->key.clear();
  }
  cudaSetDevice(cur);
  if (e != cudaSuccess) return cuda_fail(e);
  b->plan = p;
  return BZR_OK;
}

int bzr_batch_check(bzr_batch *b, void *stream, uint32_t *flags) {
  if (!b) return fail(BZR_EINVAL, "batch is null");
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  uint32_t w = 0;
  if (e == cudaSuccess)
    e = cudaMemcpy(&w, b->d_words + bzr::kNumKinds, sizeof w, cudaMemcpyDeviceToHost);
  cudaSetDevice(cur);
  if (e != cudaSuccess) return cuda_fail(e);
  if (flags) *flags = w;
  return w ? fail(BZR_EDEVICE_FLAG, "kernel bounds check fired") : BZR_OK;
}

}  // extern "C"
