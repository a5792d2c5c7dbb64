// Host interface of the traversal kernels (trace.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "layout.h"

namespace bzr {

constexpr int kTraceThreads = 128;     // default threads per block of the trace kernels
constexpr int kMaxTraceThreads = 256;  // largest block the trace kernels are compiled for
constexpr uint32_t kRayChunk = 32;     // default rays a warp takes from the global counter
constexpr int kModeFp64 = 0;   // BZR_MODE_FP64
constexpr int kModeMixed = 1;  // BZR_MODE_MIXED
// Device words launch_trace takes per call: the work counter of each kind's pass, then for
// each kind the count of rays its mixed pass deferred and the work counter of the FP64 pass
// over them.
constexpr int kTraceCounterWords = 3 * kNumKinds;

// Device pointers of one batch.  tmin / tmax may be null (0 and DBL_MAX); each output except t
// may be null.  error_word collects kErr* bits.
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
  uint32_t *error_word = nullptr;
  const uint32_t *perm = nullptr;  // optional processing order (ray indices), see RaySort
  int any_hit = 0;                 // every ray is Ray::AnyHit::yes (blazert/ray.h:24-34)
  uint32_t chunk = kRayChunk;      // rays a warp takes per fetch: 32, 64, 128, or 0 for
                                   // exactly the lanes that are idle
  uint32_t top_nodes = 0;          // top-level nodes each block stages in shared memory
  // Mixed-precision passes: rays the FP32 walk does not cover are appended to defer (one
  // word per ray of the batch, or null for launch_trace to take it from plan.pool) and traced
  // by an FP64 pass over that list right after.  Set by launch_trace.
  uint32_t *defer = nullptr;
  uint32_t *defer_count = nullptr;
  const uint32_t *n_dev = nullptr;  // when set, the pass's ray count is *n_dev (not n)
};

// Coherence sort of a batch: rays are processed in the order of a 32-bit key -- the direction
// octant (3 bits) over a Morton code of the origin quantised inside the scene bounds (9 bits
// per axis) -- bucketed on the key's top kSortBits bits by a device counting sort.  The order
// affects only speed: every ray's result is written to its own index.
struct RaySort {
  bool enabled = false;
  float lo[3] = {0, 0, 0};     // origin quantisation box
  float scale[3] = {0, 0, 0};  // 512 / extent per axis
};

// Grid of each per-kind persistent kernel: SMs x resident blocks per SM, and the launch
// shape the tuning knobs select (none of them changes results).
struct LaunchPlan {
  int sms = 0;
  int threads = kTraceThreads;     // threads per block: 64, 128 or 256
  bool shared_stack = false;       // traversal stack in shared memory even when it fits locally
  uint32_t chunk = kRayChunk;      // rays per warp fetch: 32, 64, 128 or 0 (exactly the idle lanes)
  uint32_t top_nodes = 0;          // top-level nodes each block stages in shared memory (0..256)
  // the trace kernels after a call's first one are launched with programmatic stream
  // serialisation: each is resident when its predecessor ends (it waits for it on the device)
  bool early_launch = true;
  int blocks[kNumKinds] = {0, 0, 0, 0};    // FP64 kernels
  int blocks32[kNumKinds] = {0, 0, 0, 0};  // mixed-precision kernels
  RaySort sort;
  uint32_t sort_min_rays = 1u << 16;  // smaller batches are traced in their own order
  cudaMemPool_t pool = nullptr;       // stream-ordered scratch (keeps its memory mapped)
};

// Many scenes in one launch per kind (the batching form).  Rays of scene s occupy
// [ray_offset[s], ray_offset[s+1]) of the concatenated arrays in io.  Chunks of at most
// kBatchChunk rays never cross scenes.
constexpr uint32_t kBatchChunk = 64;
struct BatchChunk {
  uint32_t scene;
  uint32_t begin, end;  // ray range in the concatenated batch
};
struct BatchView {
  const SceneView *views = nullptr;    // n_scenes device copies of the scenes' views
  const BatchChunk *chunks = nullptr;  // n_chunks
  uint32_t n_chunks = 0;
  uint32_t n_scenes = 0;
  const int8_t *first_kind = nullptr;  // per scene: kind whose pass writes the whole record
  const int8_t *last_kind = nullptr;   // per scene: kind whose pass completes the scene
  const uint32_t *scene_rays = nullptr;  // per scene: ray count
  uint32_t *scene_left = nullptr;      // per scene: rays not yet completed (set to scene_rays)
  unsigned long long *scene_done_ns = nullptr;  // per scene completion time (%globaltimer), or null
  unsigned long long *start_ns = nullptr;       // batch start time, or null
  // coherence sort of each scene's rays (BatchPlan::sort): per scene the origin quantisation
  // box, and the bits of the sort key that hold the scene index
  const RaySort *scene_sort = nullptr;
  uint32_t scene_bits = 0;
};
// Scratch of the batch coherence sort: keys and permutation (one word per ray each) and the
// 2^kSortBits bucket counts.
struct BatchSortScratch {
  uint32_t *keys = nullptr, *perm = nullptr, *counts = nullptr;
};
constexpr uint32_t kBatchSortMaxScenes = 1u << 12;  // the key keeps at least 4 bits per scene
constexpr size_t kSortBuckets = size_t(1) << 16;     // buckets of the counting sort (kSortBits)
struct BatchPlan {
  int sms = 0;
  int threads = kTraceThreads;  // threads per block: 64, 128 or 256
  bool shared_stack = false;    // traversal stack in shared memory even when it fits locally
  uint32_t local_stack = 64;    // entries of the thread-local stack: 32 or 64 (kLocalStack)
  bool sort = false;            // coherence sort of each scene's rays before tracing
  uint32_t node_width = 8;      // mixed mode: 8 walks the wide nodes, 2 the binary FP64 nodes
  int blocks[kNumKinds] = {0, 0, 0, 0};
  int blocks32[kNumKinds] = {0, 0, 0, 0};
  uint32_t stack_cap = 32;
  int kinds_present = 0;  // bit k: some scene has kind k
};
// Fills plan's grids for stack_cap, plan->threads and plan->shared_stack.
cudaError_t batch_prepare(uint32_t stack_cap, BatchPlan *plan);
// counters: kNumKinds device words (chunk counters), zeroed here.
cudaError_t launch_batch(const BatchView &B, const RayIO &io, int mode, const BatchPlan &plan,
                         cudaStream_t stream, uint32_t *counters,
                         const BatchSortScratch &sort_scratch = BatchSortScratch());

// RayHit defaults for every ray of io (a scene without primitives).
cudaError_t launch_defaults(const RayIO &io, int sms, cudaStream_t stream);

size_t trace_smem_bytes(uint32_t stack_cap, int threads);
// Dynamic shared memory of a trace_kind_kernel launch: the stack unless thread-local, then
// top_nodes staged 128-byte nodes.
size_t trace_kind_smem(uint32_t stack_cap, int threads, bool local, uint32_t top_nodes);
// Fills plan->sms and the per-kind grids for plan->threads and plan->shared_stack.
cudaError_t trace_prepare(const SceneView &S, LaunchPlan *plan);
// Number of per-kind passes a batch runs (kinds present with at least one primitive).
int trace_passes(const SceneView &S);
// Queues a batch on `stream`: one kernel per kind present, merged into io's outputs.  io.t must
// be non-null when trace_passes(S) > 1 (it carries the closest distance between passes).
// When plan.sort.enabled and the batch has at least plan.sort_min_rays rays, a coherence sort
// runs first (scratch from plan.pool, stream-ordered).
// counters: kTraceCounterWords device words, zeroed here.  totals (device, 8 x uint64, or
// null): when given, the counting kernels add per kind the box tests (totals[0..3]) and
// primitive tests (totals[4..7]) of every ray.
// A mixed-precision pass of a kind whose wide image exists is two kernels: the wide walk over
// the batch, which appends the rays its FP32 test does not cover (a direction component of 0
// or below 2^-40 in magnitude, an origin coordinate or tmin beyond 1e18, NaN) to io.defer,
// then the FP64 walk over that list.  io.defer may carry io.n words of scratch; null takes
// them from plan.pool.
cudaError_t launch_trace(const SceneView &S, const RayIO &io, int mode, const LaunchPlan &plan,
                         cudaStream_t stream, uint32_t *counters,
                         unsigned long long *totals = nullptr);

}  // namespace bzr
