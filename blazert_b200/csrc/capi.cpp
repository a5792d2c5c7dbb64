// C-ABI of libblazert_b200.so (declared in include/blazert_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "alloc.h"
#include "../../include/blazert_b200.h"
#include "layout.h"
#include "scene.h"
#include "adjoint.h"
#include "distance.h"
#include "capi_internal.h"
#include "trace.h"

namespace {

thread_local std::string g_error;

int fail(int code, const std::string &msg) {
  g_error = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char *what) {
  return fail(e == cudaErrorMemoryAllocation ? BZR_ENOMEM : BZR_ECUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

// Allocations left before the injected failure (bzr_debug_fail_allocation); 0: none armed.
std::atomic<int64_t> g_alloc_countdown{0};

// Per-call device words: kSlots slots of kSlotWords = {launch_trace's counters
// (kTraceCounterWords), error word, 3 spare}; one sticky error word for device-array calls
// follows the slots.
constexpr int kSlots = 256;
constexpr int kSlotWords = 16;
static_assert(bzr::kTraceCounterWords + 4 <= kSlotWords, "slot layout");
constexpr int kStickyWord = kSlots * kSlotWords;
// Host-array batches: split into at most host_chunks (default kHostChunks, at most kMaxChunks)
// chunks of at least host_min_chunk (default kMinChunk) rays.
constexpr int kStreams = 3;
constexpr size_t kMaxHostChunks = 32;
constexpr size_t kMaxChunks = kMaxHostChunks + 2;  // plus the two edge chunks
constexpr size_t kHostChunks = 8;
constexpr size_t kMinChunk = size_t(1) << 17;
// Host-array batches of at most kSmallBatch rays (intersect1 included) take a latency path:
// inputs packed into pinned memory, one copy in, a grid sized to the batch, one copy out.
constexpr size_t kSmallBatch = 4096;
// Collections of at least this many primitives are built on the device by default.
constexpr size_t kGpuBuildMin = size_t(1) << 16;

int default_timeout_ms() {
  const char *s = std::getenv("BZR_TIMEOUT_MS");
  const int v = s ? std::atoi(s) : 0;
  return v > 0 ? v : 600000;
}

// Bounded wait on a stream: polls cudaStreamQuery until done or the deadline passes.
int wait_stream(cudaStream_t st, int timeout_ms) {
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
  int spins = 0;
  for (;;) {
    const cudaError_t e = cudaStreamQuery(st);
    if (e == cudaSuccess) return BZR_OK;
    if (e != cudaErrorNotReady) return cuda_fail(e, "stream");
    if (timeout_ms > 0 && std::chrono::steady_clock::now() > deadline)
      return fail(BZR_ETIMEOUT, "device work did not finish within the timeout");
    if (++spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

struct bzr_scene {
  bzr::HostScene host;
  int device = -1;
  void *arena = nullptr;  // every device array of the committed scene
  bzr::SceneView view;
  bzr::AdjointView adj;
  bzr::LaunchPlan plan;
  bool sort_possible = false;  // finite scene bounds: the coherence sort can be used
  uint32_t *slots = nullptr;  // see kSlots
  std::atomic<uint32_t> next_slot{0};
  // host-pointer calls: staging buffers (grown on demand) and a private stream
  std::mutex stage_mu;
  void *stage_dev = nullptr;
  size_t stage_bytes = 0;
  uint32_t *pinned_err = nullptr;  // one error word per chunk
  unsigned char *small_pin = nullptr;  // small host-array batches: packed inputs and outputs
  cudaStream_t streams[kStreams] = {nullptr, nullptr, nullptr};
  // host-array pipeline: copies in on copy_in, kernels on streams[], copies out on copy_out,
  // chained per chunk by ev_in / ev_done
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t ev_in[kMaxChunks] = {}, ev_done[kMaxChunks] = {};
  size_t host_chunks = kHostChunks, host_min_chunk = kMinChunk;  // bzr_scene_tune
  size_t host_edge = 0;  // rays of the first and last chunk (0: all chunks the same size)
  int host_grid_div = 1;  // host-array chunks launch 1/host_grid_div of each kind's grid
  // a host-array call returned BZR_ETIMEOUT while its copies and kernels were still queued on
  // the pipeline streams, using the staging blocks (see settle_staging)
  bool stage_pending = false;

  ~bzr_scene() {
    if (device >= 0) {
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(device);
      for (cudaStream_t st : streams)
        if (st) cudaStreamSynchronize(st);
      if (copy_in) cudaStreamSynchronize(copy_in);
      if (copy_out) cudaStreamSynchronize(copy_out);
      cudaFree(arena);
      cudaFree(slots);
      cudaFree(stage_dev);
      cudaFreeHost(pinned_err);
      cudaFreeHost(small_pin);
      for (cudaStream_t st : streams)
        if (st) cudaStreamDestroy(st);
      if (copy_in) cudaStreamDestroy(copy_in);
      if (copy_out) cudaStreamDestroy(copy_out);
      for (size_t c = 0; c < kMaxChunks; ++c) {
        if (ev_in[c]) cudaEventDestroy(ev_in[c]);
        if (ev_done[c]) cudaEventDestroy(ev_done[c]);
      }
      if (plan.pool) cudaMemPoolDestroy(plan.pool);  // released once pending frees complete
      cudaSetDevice(cur);
    }
  }
};

namespace bzr {
int scene_handles(const bzr_scene *s, SceneHandles *out) {
  if (!s) return fail(BZR_EINVAL, "scene is null");
  if (!s->host.committed) return fail(BZR_ESTATE, "scene is not committed");
  out->device = s->device;
  out->view = &s->view;
  out->plan = &s->plan;
  out->error_word = s->slots + kStickyWord;
  return BZR_OK;
}
int set_error(int code, const char *msg) { return fail(code, msg); }
bool is_device_pointer(const void *p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}
}  // namespace bzr

extern "C" {

const char *bzr_last_error_string(void) { return g_error.c_str(); }

int bzr_scene_create(bzr_scene **out) {
  if (!out) return fail(BZR_EINVAL, "out is null");
  *out = new (std::nothrow) bzr_scene();
  return *out ? BZR_OK : fail(BZR_ENOMEM, "scene allocation failed");
}

int bzr_scene_destroy(bzr_scene *scene) {
  delete scene;
  return BZR_OK;
}

static int add_guard(bzr_scene *s, int kind, uint32_t *geom_id) {
  if (geom_id) *geom_id = BZR_INVALID_ID;
  if (!s) return fail(BZR_EINVAL, "scene is null");
  if (s->host.committed || s->host.kind[kind].present)
    return fail(BZR_ESTATE, "kind already added or scene already committed");
  return BZR_OK;
}

static int add_done(bzr_scene *s, int kind, uint32_t *geom_id) {
  s->host.kind[kind].present = true;
  s->host.kind[kind].geom_id = s->host.geometries++;
  if (geom_id) *geom_id = s->host.kind[kind].geom_id;
  return BZR_OK;
}

int bzr_add_mesh(bzr_scene *s, const double *v, size_t nv, const uint32_t *f, size_t nf,
                 uint32_t *geom_id) {
  int rc = add_guard(s, bzr::kMesh, geom_id);
  if (rc) return rc;
  if ((nv && !v) || (nf && !f)) return fail(BZR_EINVAL, "null mesh array");
  if (nf >= bzr::kIdMask) return fail(BZR_EINVAL, "too many faces");
  for (size_t i = 0; i < 3 * nf; ++i)
    if (f[i] >= nv) return fail(BZR_EINVAL, "face index out of range");
  try {
    bzr::add_mesh(s->host, v, nv, f, nf);
  } catch (const std::bad_alloc &) {
    return fail(BZR_ENOMEM, "host allocation failed");
  }
  return add_done(s, bzr::kMesh, geom_id);
}

int bzr_add_spheres(bzr_scene *s, const double *c, const double *r, size_t n, uint32_t *geom_id) {
  int rc = add_guard(s, bzr::kSpheres, geom_id);
  if (rc) return rc;
  if (n && (!c || !r)) return fail(BZR_EINVAL, "null sphere array");
  if (n >= bzr::kIdMask) return fail(BZR_EINVAL, "too many spheres");
  try {
    bzr::add_spheres(s->host, c, r, n);
  } catch (const std::bad_alloc &) {
    return fail(BZR_ENOMEM, "host allocation failed");
  }
  return add_done(s, bzr::kSpheres, geom_id);
}

int bzr_add_planes(bzr_scene *s, const double *c, const double *dx, const double *dy,
                   const double *rot, size_t n, uint32_t *geom_id) {
  int rc = add_guard(s, bzr::kPlanes, geom_id);
  if (rc) return rc;
  if (n && (!c || !dx || !dy || !rot)) return fail(BZR_EINVAL, "null plane array");
  if (n >= bzr::kIdMask) return fail(BZR_EINVAL, "too many planes");
  try {
    bzr::add_planes(s->host, c, dx, dy, rot, n);
  } catch (const std::bad_alloc &) {
    return fail(BZR_ENOMEM, "host allocation failed");
  }
  return add_done(s, bzr::kPlanes, geom_id);
}

int bzr_add_cylinders(bzr_scene *s, const double *c, const double *a, const double *b,
                      const double *h, const double *rot, size_t n, uint32_t *geom_id) {
  int rc = add_guard(s, bzr::kCylinders, geom_id);
  if (rc) return rc;
  if (n && (!c || !a || !b || !h || !rot)) return fail(BZR_EINVAL, "null cylinder array");
  if (n >= bzr::kIdMask) return fail(BZR_EINVAL, "too many cylinders");
  try {
    bzr::add_cylinders(s->host, c, a, b, h, rot, n);
  } catch (const std::bad_alloc &) {
    return fail(BZR_ENOMEM, "host allocation failed");
  }
  return add_done(s, bzr::kCylinders, geom_id);
}

int bzr_commit(bzr_scene *s, const bzr_build_options *options) {
  return bzr_commit_ex(s, options, 0u);
}

static int commit_scene(bzr_scene *s, uint32_t flags, bool trees_given);

int bzr_commit_ex(bzr_scene *s, const bzr_build_options *options, uint32_t flags) {
  if (!s) return fail(BZR_EINVAL, "scene is null");
  if (flags & ~uint32_t(BZR_COMMIT_GPU_BUILD | BZR_COMMIT_HOST_BUILD))
    return fail(BZR_EINVAL, "unknown commit flags");
  if ((flags & BZR_COMMIT_GPU_BUILD) && (flags & BZR_COMMIT_HOST_BUILD))
    return fail(BZR_EINVAL, "BZR_COMMIT_GPU_BUILD and BZR_COMMIT_HOST_BUILD exclude each other");
  if (s->host.committed) return fail(BZR_ESTATE, "scene already committed");
  if (options) {
    if (options->bin_size < 2 || options->max_tree_depth > 1000)
      return fail(BZR_EINVAL, "bin_size must be >= 2 and max_tree_depth <= 1000");
    s->host.opt.min_leaf = options->min_leaf_primitives;
    s->host.opt.max_depth = options->max_tree_depth;
    s->host.opt.bins = options->bin_size;
  }
  return commit_scene(s, flags, false);
}

// Builds the trees (unless trees_given: a scene read from the persistent format), flattens
// and uploads them and prepares the launch plan.
static int commit_scene(bzr_scene *s, uint32_t flags, bool trees_given) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(BZR_ENODEV, "no CUDA device");
  std::vector<bzr::KindImage> img(bzr::kNumKinds);
  uint32_t depth = 0;
  try {
    for (int k = 0; k < bzr::kNumKinds; ++k) {
      bzr::Collection &c = s->host.kind[k];
      if (!c.present) continue;
      bool built = trees_given;
      // the device build pays for its transfers and per-level launches from about 64k
      // primitives on; below that the host builds unless asked otherwise
      const bool want_gpu = (flags & BZR_COMMIT_GPU_BUILD) ||
                            (!(flags & BZR_COMMIT_HOST_BUILD) && c.boxes.n >= kGpuBuildMin);
      if (!built && want_gpu && bzr::gpu_build_possible(c.boxes, s->host.opt)) {
        const auto t0 = std::chrono::steady_clock::now();
        bzr::Tree t;
        if (bzr::gpu_build_tree(c.boxes, s->host.opt, &t) == cudaSuccess) {
          t.build_seconds =
              std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
          c.tree = std::move(t);
          built = true;
        } else {
          cudaGetLastError();  // clear a launch error; the host builds the same tree
        }
      }
      if (!built) c.tree = bzr::build_tree(c.boxes, s->host.opt);
      depth = std::max(depth, c.tree.max_depth);
      img[k] = bzr::flatten(s->host, k);
    }
  } catch (const std::bad_alloc &) {
    return fail(BZR_ENOMEM, "host allocation failed during the build");
  }
  // One device arena holds every array, each 256-byte aligned.
  struct Piece {
    const void *src;
    size_t bytes;
    size_t off;
  };
  std::vector<Piece> pieces;
  size_t total = 0;
  auto place = [&](const void *src, size_t bytes) {
    const size_t off = total;
    pieces.push_back({src, bytes, off});
    total = align_up(total + std::max<size_t>(bytes, 1), 256);
    return off;
  };
  size_t off_nodes64[4], off_wide[4], off_leaves[4], off_payload[4], off_ids[4], off_tri[4],
      off_tv[4], off_pos[4], off_vnorm[4];
  uint32_t wide_stack = 0;
  for (int k = 0; k < bzr::kNumKinds; ++k) {
    off_nodes64[k] = place(img[k].nodes64.data(), img[k].nodes64.size() * sizeof(double));
    off_wide[k] = place(img[k].wide.data(), img[k].wide.size());
    off_leaves[k] = place(img[k].leaves.data(), img[k].leaves.size() * sizeof(double));
    if (img[k].mixed_ok) wide_stack = std::max(wide_stack, img[k].wide_stack);
    off_payload[k] = place(img[k].payload.data(), img[k].payload.size() * sizeof(double));
    off_ids[k] = place(img[k].prim_ids.data(), img[k].prim_ids.size() * sizeof(uint32_t));
    off_pos[k] = place(img[k].pos_of.data(), img[k].pos_of.size() * sizeof(uint32_t));
    off_tri[k] = place(img[k].tri.data(), img[k].tri.size() * sizeof(uint32_t));
    off_tv[k] = place(img[k].verts.data(), img[k].verts.size() * sizeof(double));
    off_vnorm[k] = place(img[k].vnorm.data(), img[k].vnorm.size() * sizeof(double));
  }
  const size_t off_faces = place(s->host.faces.data(), s->host.faces.size() * sizeof(uint32_t));
  const size_t off_vn = place(s->host.vert_n.data(), s->host.vert_n.size() * sizeof(double));
  // input-order geometry for the adjoint
  const size_t off_verts =
      place(s->host.vertices.data(), s->host.vertices.size() * sizeof(double));
  const bzr::Collection &sph = s->host.kind[bzr::kSpheres];
  const size_t off_sc = place(sph.a.data(), sph.a.size() * sizeof(double));
  const size_t off_sr = place(sph.b.data(), sph.b.size() * sizeof(double));
  // A commit that failed after its first device allocation leaves the scene uncommitted with
  // those allocations held: free them before this attempt allocates its own.
  if (s->arena) cudaFree(s->arena);
  if (s->slots) cudaFree(s->slots);
  if (s->pinned_err) cudaFreeHost(s->pinned_err);
  if (s->plan.pool) cudaMemPoolDestroy(s->plan.pool);
  s->arena = nullptr;
  s->slots = nullptr;
  s->pinned_err = nullptr;
  s->plan.pool = nullptr;
  cudaError_t e = cudaGetDevice(&s->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  e = bzr::dev_malloc(&s->arena, total);
  if (e != cudaSuccess) return fail(BZR_ENOMEM, "device arena allocation failed");
  for (const Piece &p : pieces) {
    if (!p.bytes) continue;
    e = cudaMemcpy(static_cast<char *>(s->arena) + p.off, p.src, p.bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "scene upload");
  }
  char *base = static_cast<char *>(s->arena);
  for (int k = 0; k < bzr::kNumKinds; ++k) {
    bzr::KindView &v = s->view.k[k];
    const bzr::Collection &c = s->host.kind[k];
    v.present = c.present ? 1 : 0;
    v.geom_id = c.geom_id;
    if (!c.present) continue;
    v.nodes64 = reinterpret_cast<const double *>(base + off_nodes64[k]);
    v.wide = reinterpret_cast<const unsigned char *>(base + off_wide[k]);
    v.leaves = reinterpret_cast<const double *>(base + off_leaves[k]);
    v.n_wide = img[k].n_wide;
    v.n_leaf16 = img[k].n_leaf16;
    v.wide_root_ref = img[k].wide_root_ref;
    v.payload = reinterpret_cast<const double *>(base + off_payload[k]);
    v.prim_ids = reinterpret_cast<const uint32_t *>(base + off_ids[k]);
    v.pos_of = reinterpret_cast<const uint32_t *>(base + off_pos[k]);
    v.tri = reinterpret_cast<const uint32_t *>(base + off_tri[k]);
    v.verts = reinterpret_cast<const double *>(base + off_tv[k]);
    v.vnorm = reinterpret_cast<const double *>(base + off_vnorm[k]);
    v.n_internal = img[k].n_internal;
    v.n_prims = static_cast<uint32_t>(img[k].prim_ids.size());
    v.n_verts = static_cast<uint32_t>(img[k].verts.size() / bzr::kVertexDoubles);
    v.root_ref = img[k].root_ref;
    v.mixed_ok = img[k].mixed_ok ? 1 : 0;
    std::memcpy(v.root_box, img[k].root_box, sizeof v.root_box);
    v.coord_max = img[k].coord_max;
  }
  s->view.faces = reinterpret_cast<const uint32_t *>(base + off_faces);
  s->view.vert_n = reinterpret_cast<const double *>(base + off_vn);
  if (s->host.kind[bzr::kMesh].present) {
    s->adj.verts = reinterpret_cast<const double *>(base + off_verts);
    s->adj.faces = s->view.faces;
    s->adj.vert_n = s->view.vert_n;
    s->adj.n_faces = s->host.faces.size() / 3;
    s->adj.mesh_geom = s->host.kind[bzr::kMesh].geom_id;
  }
  if (sph.present) {
    s->adj.centers = reinterpret_cast<const double *>(base + off_sc);
    s->adj.radii = reinterpret_cast<const double *>(base + off_sr);
    s->adj.sphere_geom = sph.geom_id;
  }
  s->view.stack_cap = std::max<uint32_t>({8, depth + 2, wide_stack});
  e = bzr::dev_malloc(&s->slots, (kStickyWord + 1) * sizeof(uint32_t));
  if (e != cudaSuccess) return fail(BZR_ENOMEM, "slot allocation failed");
  e = cudaMemset(s->slots, 0, (kStickyWord + 1) * sizeof(uint32_t));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemset");
  e = bzr::host_malloc(&s->pinned_err, kMaxChunks * sizeof(uint32_t));
  if (e != cudaSuccess) return fail(BZR_ENOMEM, "pinned allocation failed");
  e = bzr::trace_prepare(s->view, &s->plan);
  if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
  {  // per-scene memory pool for per-call scratch; it keeps freed memory for reuse
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->device;
    e = cudaMemPoolCreate(&s->plan.pool, &props);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemPoolCreate");
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(s->plan.pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemPoolSetAttribute");
  }
  {  // origin quantisation box of the coherence sort: union of the per-kind root boxes
    double lo[3] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max(),
                    std::numeric_limits<double>::max()};
    double hi[3] = {-lo[0], -lo[1], -lo[2]};
    for (int k = 0; k < bzr::kNumKinds; ++k) {
      const bzr::KindView &v = s->view.k[k];
      if (!v.present || !v.n_prims) continue;
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], v.root_box[2 * a]);
        hi[a] = std::max(hi[a], v.root_box[2 * a + 1]);
      }
    }
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      const double ext = hi[a] - lo[a];
      ok = ok && std::isfinite(ext) && std::abs(lo[a]) < 1e30 && std::abs(hi[a]) < 1e30;
      s->plan.sort.lo[a] = static_cast<float>(lo[a]);
      s->plan.sort.scale[a] = ext > 0 ? static_cast<float>(512.0 / ext) : 0.0f;
    }
    // Off by default: on the B200 the coherent order made the trace kernels slower on every
    // workload measured (heightfield 3.37 vs 3.05 ms per launch, icosphere 620 vs 389 us);
    // blazert_b200.autotune switches it on where it pays.
    s->plan.sort.enabled = false;
    s->sort_possible = ok;
  }
  s->host.committed = true;
  return BZR_OK;
}

static bool is_device_ptr(const void *p) { return bzr::is_device_pointer(p); }

// The host-array pipeline's streams and events, made on the first host-array call (scenes
// only queried with device arrays, or through a batch, never need them).  The caller holds
// stage_mu.
static cudaError_t make_pipeline(bzr_scene *s) {
  if (s->copy_out) return cudaSuccess;
  cudaError_t ce = cudaSuccess;
  for (cudaStream_t &st : s->streams)
    if (ce == cudaSuccess && !st) ce = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  for (size_t c = 0; c < kMaxChunks && ce == cudaSuccess; ++c) {
    if (!s->ev_in[c]) ce = cudaEventCreateWithFlags(&s->ev_in[c], cudaEventDisableTiming);
    if (ce == cudaSuccess && !s->ev_done[c])
      ce = cudaEventCreateWithFlags(&s->ev_done[c], cudaEventDisableTiming);
  }
  if (ce == cudaSuccess && !s->copy_in)
    ce = cudaStreamCreateWithFlags(&s->copy_in, cudaStreamNonBlocking);
  // copy_out last: its presence marks the whole set as made
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&s->copy_out, cudaStreamNonBlocking);
  return ce;
}

// Waits for a stream: spins on cudaStreamQuery for up to spin_us (a small batch finishes in
// tens of microseconds, well inside a sleeping wait's granularity), then waits as usual.
static int wait_stream_spin(cudaStream_t st, int spin_us) {
  const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(spin_us);
  do {
    const cudaError_t e = cudaStreamQuery(st);
    if (e == cudaSuccess) return BZR_OK;
    if (e != cudaErrorNotReady) return cuda_fail(e, "stream");
  } while (std::chrono::steady_clock::now() < until);
  return wait_stream(st, default_timeout_ms());
}

// A host-array call that timed out left its copies and kernels queued on the pipeline streams,
// still reading and writing the staging blocks.  Before a later call reuses them, every
// pipeline stream must have finished; if one is still busy after the bounded wait, that call
// times out too and the staging stays reserved.  The caller holds stage_mu.
static int settle_staging(bzr_scene *s) {
  if (!s->stage_pending) return BZR_OK;
  for (cudaStream_t q : {s->copy_in, s->streams[0], s->streams[1], s->streams[2], s->copy_out}) {
    if (!q) continue;
    const int rc = wait_stream(q, default_timeout_ms());
    if (rc) return rc;
  }
  s->stage_pending = false;
  return BZR_OK;
}

// Return code of a wait on queued host-array work; a timeout marks the staging as still in use.
static int staged_wait_result(bzr_scene *s, int rc) {
  if (rc == BZR_ETIMEOUT) s->stage_pending = true;
  return rc;
}

// The latency path of small host-array batches (the caller holds stage_mu).  One pinned block
// mirrors one device block: inputs org, dir, [tmin], [tmax]; then the error word; then the
// outputs t, [uv], [normal], [prim], [geom], [hit]; each piece 256-byte aligned.  One copy in,
// the kind passes on a grid sized to the batch, one copy out, the outputs unpacked on the host.
static int run_small(bzr_scene *s, size_t n, const double *org, const double *dir,
                     const double *tmin, const double *tmax, double *t, double *uv, double *normal,
                     uint32_t *prim, uint32_t *geom, uint8_t *hit, int mode, bzr::RayIO io,
                     uint32_t *counters, unsigned long long *totals) {
  struct Piece {
    size_t bytes, off;
  };
  size_t total = 0;
  auto place = [&](size_t bytes) {
    const Piece p{bytes, total};
    total += align_up(bytes ? bytes : 0, 256);
    return p;
  };
  const Piece p_org = place(24 * n), p_dir = place(24 * n), p_tmin = place(tmin ? 8 * n : 0),
              p_tmax = place(tmax ? 8 * n : 0), p_err = place(sizeof(uint32_t));
  const size_t in_bytes = total;
  const Piece p_t = place(8 * n), p_uv = place(uv ? 16 * n : 0), p_n = place(normal ? 24 * n : 0),
              p_prim = place(prim ? 4 * n : 0), p_geom = place(geom ? 4 * n : 0),
              p_hit = place(hit ? n : 0);
  const size_t out_begin = p_t.off, out_bytes = total - out_begin;
  // the block for kSmallBatch rays with every piece bounds what any small batch needs
  const size_t cap = 8 * align_up(24 * kSmallBatch, 256) + 256;
  if (!s->small_pin && bzr::host_malloc(&s->small_pin, cap) != cudaSuccess) {
    s->small_pin = nullptr;
    return fail(BZR_ENOMEM, "pinned staging allocation failed");
  }
  if (s->stage_bytes < cap) {
    cudaFree(s->stage_dev);
    s->stage_dev = nullptr;
    s->stage_bytes = 0;
    if (bzr::dev_malloc(&s->stage_dev, cap) != cudaSuccess)
      return fail(BZR_ENOMEM, "staging allocation failed");
    s->stage_bytes = cap;
  }
  unsigned char *h = s->small_pin;
  auto *d = static_cast<unsigned char *>(s->stage_dev);
  std::memcpy(h + p_org.off, org, p_org.bytes);
  std::memcpy(h + p_dir.off, dir, p_dir.bytes);
  if (tmin) std::memcpy(h + p_tmin.off, tmin, p_tmin.bytes);
  if (tmax) std::memcpy(h + p_tmax.off, tmax, p_tmax.bytes);
  std::memset(h + p_err.off, 0, sizeof(uint32_t));
  cudaStream_t st = s->streams[0];
  bzr::RayIO ci = io;
  ci.org = reinterpret_cast<const double *>(d + p_org.off);
  ci.dir = reinterpret_cast<const double *>(d + p_dir.off);
  ci.tmin = tmin ? reinterpret_cast<const double *>(d + p_tmin.off) : nullptr;
  ci.tmax = tmax ? reinterpret_cast<const double *>(d + p_tmax.off) : nullptr;
  ci.error_word = reinterpret_cast<uint32_t *>(d + p_err.off);
  ci.t = reinterpret_cast<double *>(d + p_t.off);
  ci.uv = uv ? reinterpret_cast<double *>(d + p_uv.off) : nullptr;
  ci.normal = normal ? reinterpret_cast<double *>(d + p_n.off) : nullptr;
  ci.prim = prim ? reinterpret_cast<uint32_t *>(d + p_prim.off) : nullptr;
  ci.geom = geom ? reinterpret_cast<uint32_t *>(d + p_geom.off) : nullptr;
  ci.hit = hit ? reinterpret_cast<uint8_t *>(d + p_hit.off) : nullptr;
  bzr::LaunchPlan plan = s->plan;
  const int need_blocks = static_cast<int>((n + plan.threads - 1) / plan.threads);
  for (int k = 0; k < bzr::kNumKinds; ++k) {
    plan.blocks[k] = std::max(1, std::min(plan.blocks[k], need_blocks));
    plan.blocks32[k] = std::max(1, std::min(plan.blocks32[k], need_blocks));
  }
  cudaError_t e = cudaMemcpyAsync(d, h, in_bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = bzr::launch_trace(s->view, ci, mode, plan, st, counters, totals);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h + out_begin, d + out_begin, out_bytes, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h + p_err.off, d + p_err.off, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return cuda_fail(e, "small batch submission");
  const int rc = staged_wait_result(s, wait_stream_spin(st, 2000));
  if (rc) return rc;
  if (t) std::memcpy(t, h + p_t.off, p_t.bytes);
  if (uv) std::memcpy(uv, h + p_uv.off, p_uv.bytes);
  if (normal) std::memcpy(normal, h + p_n.off, p_n.bytes);
  if (prim) std::memcpy(prim, h + p_prim.off, p_prim.bytes);
  if (geom) std::memcpy(geom, h + p_geom.off, p_geom.bytes);
  if (hit) std::memcpy(hit, h + p_hit.off, p_hit.bytes);
  uint32_t bits = 0;
  std::memcpy(&bits, h + p_err.off, sizeof bits);
  if (bits)
    return fail(BZR_EDEVICE_FLAG, "kernel bounds check fired (error bits " +
                                      std::to_string(bits) + ")");
  return BZR_OK;
}

// Shared body of bzr_intersectN and bzr_work_counts; totals (device) selects the counting
// kernel.
static int run_batch(const bzr_scene *cs, size_t n, const double *org, const double *dir,
                     const double *tmin, const double *tmax, double *t, double *uv,
                     double *normal, uint32_t *prim, uint32_t *geom, uint8_t *hit, int mode,
                     uint32_t ray_flags, void *stream, unsigned long long *totals) {
  bzr_scene *s = const_cast<bzr_scene *>(cs);
  if (!s) return fail(BZR_EINVAL, "scene is null");
  if (!s->host.committed) return fail(BZR_ESTATE, "scene is not committed");
  if (mode != BZR_MODE_FP64 && mode != BZR_MODE_MIXED) return fail(BZR_EINVAL, "bad mode");
  if (ray_flags & ~uint32_t(BZR_RAY_ANY_HIT)) return fail(BZR_EINVAL, "unknown ray flags");
  if (n == 0) return BZR_OK;
  if (!org || !dir) return fail(BZR_EINVAL, "origins and directions are required");
  if (n > 0x7FFFFFC0u) return fail(BZR_EINVAL, "batch too large (at most 2^31 - 64 rays)");
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != s->device) cudaSetDevice(s->device);
  struct DevGuard {
    int d;
    ~DevGuard() { cudaSetDevice(d); }
  } guard{cur};

  const void *ptrs[10] = {org, dir, tmin, tmax, t, uv, normal, prim, geom, hit};
  int n_dev = 0, n_given = 0;
  for (const void *p : ptrs)
    if (p) {
      ++n_given;
      n_dev += is_device_ptr(p) ? 1 : 0;
    }
  const uint32_t slot = s->next_slot.fetch_add(1) % kSlots;
  uint32_t *counters = s->slots + kSlotWords * slot;
  bzr::RayIO io;
  io.n = static_cast<uint32_t>(n);
  io.any_hit = (ray_flags & BZR_RAY_ANY_HIT) ? 1 : 0;

  if (n_dev == n_given) {  // device arrays: queue on the caller's stream and return
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    io.org = org; io.dir = dir; io.tmin = tmin; io.tmax = tmax;
    io.t = t; io.uv = uv; io.normal = normal; io.prim = prim; io.geom = geom; io.hit = hit;
    io.error_word = s->slots + kStickyWord;  // sticky, read by bzr_scene_check
    cudaError_t e = cudaSuccess;
    if (!t) {  // the passes carry the closest distance in t: stream-ordered scratch
      e = bzr::pool_malloc(&io.t, 8 * n, s->plan.pool, st);
      if (e != cudaSuccess) return fail(BZR_ENOMEM, "distance scratch allocation failed");
    }
    e = bzr::launch_trace(s->view, io, mode, s->plan, st, counters, totals);
    if (!t) cudaFreeAsync(io.t, st);
    return e == cudaSuccess ? BZR_OK : cuda_fail(e, "kernel launch");
  }
  if (n_dev != 0) return fail(BZR_EINVAL, "arrays must be all host or all device memory");

  // Host arrays: stage through device buffers on the scene's stream.
  std::lock_guard<std::mutex> lock(s->stage_mu);
  if (const cudaError_t ce = make_pipeline(s)) return cuda_fail(ce, "cudaStreamCreate");
  if (const int rc = settle_staging(s)) return rc;
  if (n <= kSmallBatch)
    return run_small(s, n, org, dir, tmin, tmax, t, uv, normal, prim, geom, hit, mode, io,
                     counters, totals);
  // every staged array starts on a 256-byte boundary (see take() below)
  const size_t piece_bytes[10] = {24 * n, 24 * n, tmin ? 8 * n : 0, tmax ? 8 * n : 0,
                                  8 * n, uv ? 16 * n : 0, normal ? 24 * n : 0,
                                  prim ? 4 * n : 0, geom ? 4 * n : 0, hit ? n : 0};
  size_t need = 0;
  for (size_t b : piece_bytes)
    if (b) need += align_up(b, 256);
  if (s->stage_bytes < need) {
    cudaFree(s->stage_dev);
    s->stage_dev = nullptr;
    s->stage_bytes = 0;
    if (bzr::dev_malloc(&s->stage_dev, need) != cudaSuccess)
      return fail(BZR_ENOMEM, "staging allocation failed");
    s->stage_bytes = need;
  }
  char *p = static_cast<char *>(s->stage_dev);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char *q = p + off;
    off = align_up(off + bytes, 256);
    return q;
  };
  double *d_org = reinterpret_cast<double *>(take(24 * n));
  double *d_dir = reinterpret_cast<double *>(take(24 * n));
  double *d_tmin = tmin ? reinterpret_cast<double *>(take(8 * n)) : nullptr;
  double *d_tmax = tmax ? reinterpret_cast<double *>(take(8 * n)) : nullptr;
  double *d_t = reinterpret_cast<double *>(take(8 * n));  // always: the passes carry the distance
  double *d_uv = uv ? reinterpret_cast<double *>(take(16 * n)) : nullptr;
  double *d_normal = normal ? reinterpret_cast<double *>(take(24 * n)) : nullptr;
  uint32_t *d_prim = prim ? reinterpret_cast<uint32_t *>(take(4 * n)) : nullptr;
  uint32_t *d_geom = geom ? reinterpret_cast<uint32_t *>(take(4 * n)) : nullptr;
  uint8_t *d_hit = hit ? reinterpret_cast<uint8_t *>(take(n)) : nullptr;
  // A three-stage pipeline over chunks: the copies in run ahead on copy_in, each chunk's
  // kernels start on one of the scene's streams (round robin, so that one chunk's slowest rays
  // overlap the next chunk's kernels) once its copies in are done, and its copies out follow
  // on copy_out once its kernels are done.
  // The kernels are the slowest stage, so a step takes about the first chunk's copy in, the
  // kernels of every chunk and the last chunk's copy out: optional small edge chunks shorten
  // the exposed copies, a few large middle chunks keep the kernels' per-launch tails few.
  size_t bounds[kMaxChunks + 1];
  size_t nchunks = 0;
  {
    const size_t edge = s->host_edge, min_chunk = s->host_min_chunk, max_chunks = s->host_chunks;
    const bool edges = edge > 0 && n > 4 * edge;
    const size_t first = edges ? edge : 0, mid = n - 2 * first;
    const size_t chunk =
        mid <= min_chunk ? mid : std::max(min_chunk, (mid + max_chunks - 1) / max_chunks);
    bounds[0] = 0;
    if (edges) bounds[++nchunks] = first;
    for (size_t a = first; a < first + mid; a += chunk) bounds[++nchunks] = std::min(first + mid, a + chunk);
    if (edges) bounds[++nchunks] = n;
  }
  // chunks on the round-robin streams may run side by side on smaller grids, so that one
  // chunk's tail idles only its share of the SMs
  bzr::LaunchPlan chunk_plan = s->plan;
  // chunks run on several streams at once: a pass's blocks that wait in place for the previous
  // pass would hold SMs that another chunk's kernels could use
  chunk_plan.early_launch = false;
  for (int k = 0; k < bzr::kNumKinds; ++k) {
    chunk_plan.blocks[k] = std::max(1, chunk_plan.blocks[k] / s->host_grid_div);
    chunk_plan.blocks32[k] = std::max(1, chunk_plan.blocks32[k] / s->host_grid_div);
  }
  cudaError_t e = cudaSuccess;
  for (size_t c = 0; c < nchunks && e == cudaSuccess; ++c) {
    const size_t a = bounds[c], m = bounds[c + 1] - a;
    cudaStream_t st = s->streams[c % kStreams];
    uint32_t *cnt = c == 0 ? counters : s->slots + kSlotWords * (s->next_slot.fetch_add(1) % kSlots);
    auto h2d = [&](double *dst, const double *src, size_t per) {
      if (src && e == cudaSuccess)
        e = cudaMemcpyAsync(dst + per * a, src + per * a, 8 * per * m, cudaMemcpyHostToDevice,
                            s->copy_in);
    };
    h2d(d_org, org, 3);
    h2d(d_dir, dir, 3);
    h2d(d_tmin, tmin, 1);
    h2d(d_tmax, tmax, 1);
    bzr::RayIO ci;
    ci.n = static_cast<uint32_t>(m);
    ci.any_hit = io.any_hit;
    ci.org = d_org + 3 * a;
    ci.dir = d_dir + 3 * a;
    ci.tmin = d_tmin ? d_tmin + a : nullptr;
    ci.tmax = d_tmax ? d_tmax + a : nullptr;
    ci.t = d_t + a;
    ci.uv = d_uv ? d_uv + 2 * a : nullptr;
    ci.normal = d_normal ? d_normal + 3 * a : nullptr;
    ci.prim = d_prim ? d_prim + a : nullptr;
    ci.geom = d_geom ? d_geom + a : nullptr;
    ci.hit = d_hit ? d_hit + a : nullptr;
    ci.error_word = cnt + bzr::kTraceCounterWords;
    if (e == cudaSuccess) e = cudaEventRecord(s->ev_in[c], s->copy_in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, s->ev_in[c], 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(ci.error_word, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess) e = bzr::launch_trace(s->view, ci, mode, chunk_plan, st, cnt, totals);
    if (e == cudaSuccess) e = cudaEventRecord(s->ev_done[c], st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->copy_out, s->ev_done[c], 0);
    auto d2h = [&](void *dst, const void *src, size_t bytes) {
      if (dst && e == cudaSuccess)
        e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->copy_out);
    };
    d2h(t ? t + a : nullptr, ci.t, 8 * m);
    d2h(uv ? uv + 2 * a : nullptr, ci.uv, 16 * m);
    d2h(normal ? normal + 3 * a : nullptr, ci.normal, 24 * m);
    d2h(prim ? prim + a : nullptr, ci.prim, 4 * m);
    d2h(geom ? geom + a : nullptr, ci.geom, 4 * m);
    d2h(hit ? hit + a : nullptr, ci.hit, m);
    d2h(s->pinned_err + c, ci.error_word, sizeof(uint32_t));
  }
  if (e != cudaSuccess) return cuda_fail(e, "batch submission");
  for (cudaStream_t q : {s->copy_in, s->streams[0], s->streams[1], s->streams[2], s->copy_out}) {
    const int rc = staged_wait_result(s, wait_stream(q, default_timeout_ms()));
    if (rc) return rc;
  }
  uint32_t bits = 0;
  for (size_t c = 0; c < nchunks; ++c) bits |= s->pinned_err[c];
  if (bits)
    return fail(BZR_EDEVICE_FLAG, "kernel bounds check fired (error bits " +
                                      std::to_string(bits) + ")");
  return BZR_OK;
}

int bzr_intersectN(const bzr_scene *s, size_t n, const double *org, const double *dir,
                   const double *tmin, const double *tmax, double *t, double *uv, double *normal,
                   uint32_t *prim, uint32_t *geom, uint8_t *hit, int mode, void *stream) {
  return run_batch(s, n, org, dir, tmin, tmax, t, uv, normal, prim, geom, hit, mode, 0u, stream,
                   nullptr);
}

int bzr_intersectN_ex(const bzr_scene *s, size_t n, const double *org, const double *dir,
                      const double *tmin, const double *tmax, double *t, double *uv,
                      double *normal, uint32_t *prim, uint32_t *geom, uint8_t *hit, int mode,
                      uint32_t ray_flags, void *stream) {
  return run_batch(s, n, org, dir, tmin, tmax, t, uv, normal, prim, geom, hit, mode, ray_flags,
                   stream, nullptr);
}

int bzr_work_counts(const bzr_scene *cs, size_t n, const double *org, const double *dir,
                    const double *tmin, const double *tmax, uint64_t totals[8], void *stream) {
  if (!totals) return fail(BZR_EINVAL, "null argument");
  uint64_t all[16];
  const int rc = bzr_work_counts_ex(cs, n, org, dir, tmin, tmax, BZR_MODE_FP64, all, stream);
  for (int k = 0; k < 8; ++k) totals[k] = rc == BZR_OK ? all[k] : 0;
  return rc;
}

int bzr_work_counts_ex(const bzr_scene *cs, size_t n, const double *org, const double *dir,
                       const double *tmin, const double *tmax, int mode, uint64_t totals[16],
                       void *stream) {
  bzr_scene *s = const_cast<bzr_scene *>(cs);
  if (!s || !totals) return fail(BZR_EINVAL, "null argument");
  if (!s->host.committed) return fail(BZR_ESTATE, "scene is not committed");
  if (mode != BZR_MODE_FP64 && mode != BZR_MODE_MIXED) return fail(BZR_EINVAL, "bad mode");
  for (int k = 0; k < 16; ++k) totals[k] = 0;
  if (n == 0) return BZR_OK;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(s->device);
  unsigned long long *dev = nullptr;
  cudaError_t e = bzr::dev_malloc(&dev, 16 * sizeof(unsigned long long));
  if (e != cudaSuccess) {
    cudaSetDevice(cur);
    return fail(BZR_ENOMEM, "counter allocation failed");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  e = cudaMemsetAsync(dev, 0, 16 * sizeof(unsigned long long), st);
  int rc = e == cudaSuccess ? BZR_OK : cuda_fail(e, "cudaMemsetAsync");
  cudaSetDevice(cur);
  if (rc == BZR_OK)
    rc = run_batch(s, n, org, dir, tmin, tmax, nullptr, nullptr, nullptr, nullptr, nullptr,
                   nullptr, mode, 0u, stream, dev);
  cudaSetDevice(s->device);
  // the host path ran on the scene's streams; make the counter copy wait for all of them
  for (cudaStream_t q : s->streams)
    if (rc == BZR_OK) rc = wait_stream(q, default_timeout_ms());
  if (rc == BZR_OK) rc = wait_stream(st, default_timeout_ms());
  if (rc == BZR_OK) {
    unsigned long long h[16];
    e = cudaMemcpy(h, dev, sizeof h, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
      rc = cuda_fail(e, "counter read");
    else
      for (int k = 0; k < 16; ++k) totals[k] = h[k];
  }
  cudaFree(dev);
  cudaSetDevice(cur);
  return rc;
}

int bzr_adjoint_hit(const bzr_scene *cs, size_t n, const double *origins,
                    const double *directions, const double *hit_distance, const uint32_t *prim_id,
                    const uint32_t *geom_id, const uint8_t *hit, const double *grad_t,
                    const double *grad_uv, const double *grad_normal, double *grad_vertices,
                    double *grad_centers, double *grad_radii, double *grad_origins,
                    double *grad_directions, void *stream) {
  bzr_scene *s = const_cast<bzr_scene *>(cs);
  if (!s) return fail(BZR_EINVAL, "scene is null");
  if (!s->host.committed) return fail(BZR_ESTATE, "scene is not committed");
  if (n == 0) return BZR_OK;
  if (!origins || !directions || !hit_distance || !prim_id || !geom_id || !hit)
    return fail(BZR_EINVAL, "forward results are required");
  const void *ptrs[] = {origins, directions, hit_distance, prim_id, geom_id, hit, grad_t,
                        grad_uv, grad_normal, grad_vertices, grad_centers, grad_radii,
                        grad_origins, grad_directions};
  for (const void *p : ptrs)
    if (p && !is_device_ptr(p)) return fail(BZR_EINVAL, "adjoint arrays must be device memory");
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(s->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  bzr::AdjointIO io;
  io.n = n;
  io.org = origins;
  io.dir = directions;
  io.t = hit_distance;
  io.prim = prim_id;
  io.geom = geom_id;
  io.hit = hit;
  io.grad_t = grad_t;
  io.grad_uv = grad_uv;
  io.grad_normal = grad_normal;
  io.grad_verts = grad_vertices;
  io.grad_centers = grad_centers;
  io.grad_radii = grad_radii;
  io.grad_org = grad_origins;
  io.grad_dir = grad_directions;
  io.error_word = s->slots + kStickyWord;
  const size_t nv = s->host.vertices.size() / 3, ns = s->host.kind[bzr::kSpheres].n;
  cudaError_t e = cudaSuccess;
  if (grad_vertices) e = cudaMemsetAsync(grad_vertices, 0, 24 * nv, st);
  if (e == cudaSuccess && grad_centers) e = cudaMemsetAsync(grad_centers, 0, 24 * ns, st);
  if (e == cudaSuccess && grad_radii) e = cudaMemsetAsync(grad_radii, 0, 8 * ns, st);
  double *gvn = nullptr;
  if (e == cudaSuccess && grad_vertices && nv) {
    e = bzr::pool_malloc(&gvn, 24 * nv, s->plan.pool, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(gvn, 0, 24 * nv, st);
  }
  io.grad_vert_n = gvn;
  if (e == cudaSuccess) e = bzr::launch_adjoint(s->adj, io, s->plan.sms, st);
  if (gvn) cudaFreeAsync(gvn, st);
  cudaSetDevice(cur);
  return e == cudaSuccess ? BZR_OK : cuda_fail(e, "adjoint launch");
}

// Shared body of the two distance queries: kind >= 0 is the per-primitive form, -1 the scene
// form.  Device arrays are queued on the caller's stream; host arrays are staged through
// stream-ordered scratch from the scene's pool and the call waits for the results.
static int run_distance(const bzr_scene *cs, int kind, size_t n, const uint32_t *ids,
                        const double *points, double *distance, double *closest, uint32_t *prim,
                        uint32_t *geom, void *stream) {
  bzr_scene *s = const_cast<bzr_scene *>(cs);
  if (!s) return fail(BZR_EINVAL, "scene is null");
  if (!s->host.committed) return fail(BZR_ESTATE, "scene is not committed");
  if (kind >= bzr::kNumKinds || kind < -1) return fail(BZR_EINVAL, "bad primitive kind");
  if (kind >= 0 && !s->host.kind[kind].present)
    return fail(BZR_EINVAL, "the scene has no primitives of this kind");
  if (closest && kind != bzr::kMesh)
    return fail(BZR_EINVAL, "closest points are returned for triangles only");
  if (n == 0) return BZR_OK;
  if (!points || !distance || (kind >= 0 && !ids)) return fail(BZR_EINVAL, "null argument");
  if (n > (size_t(1) << 40)) return fail(BZR_EINVAL, "batch too large");
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != s->device) cudaSetDevice(s->device);
  struct DevGuard {
    int d;
    ~DevGuard() { cudaSetDevice(d); }
  } guard{cur};
  const void *ptrs[6] = {ids, points, distance, closest, prim, geom};
  int n_dev = 0, n_given = 0;
  for (const void *p : ptrs)
    if (p) {
      ++n_given;
      n_dev += is_device_ptr(p) ? 1 : 0;
    }
  if (n_dev != 0 && n_dev != n_given)
    return fail(BZR_EINVAL, "arrays must be all host or all device memory");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  bzr::DistanceIO io;
  io.n = n;
  io.error_word = s->slots + kStickyWord;
  auto launch = [&]() {
    return kind >= 0 ? bzr::launch_distance(s->view, kind, io, s->plan.sms, st)
                     : bzr::launch_nearest(s->view, io, s->plan.sms, s->plan.pool, st);
  };
  if (n_dev == n_given) {
    io.ids = ids; io.points = points; io.distance = distance; io.closest = closest;
    io.prim = prim; io.geom = geom;
    const cudaError_t e = launch();
    return e == cudaSuccess ? BZR_OK : cuda_fail(e, "distance launch");
  }
  // Host arrays: the ray path's three-stage pipeline over chunks -- copies in on copy_in,
  // each chunk's kernel on one of the scene's streams once its copies are in, copies out on
  // copy_out once its kernel is done -- with stream-ordered staging from the scene's pool.
  std::lock_guard<std::mutex> lock(s->stage_mu);
  if (const cudaError_t ce = make_pipeline(s)) return cuda_fail(ce, "cudaStreamCreate");
  if (const int rc = settle_staging(s)) return rc;
  // bytes per query of each staged array: ids, points | distance, closest, prim, geom
  const size_t per[6] = {kind >= 0 ? 4u : 0u, 24, 8, closest ? 24u : 0u, prim ? 4u : 0u,
                         geom ? 4u : 0u};
  size_t total = 256;  // the call's own error word first (ids outside the kind)
  for (size_t b : per) total += align_up(b * n, 256);
  char *dev = nullptr;
  cudaError_t e =
      bzr::pool_malloc(&dev, total, s->plan.pool, s->copy_in);
  if (e != cudaSuccess) return fail(BZR_ENOMEM, "distance staging allocation failed");
  uint32_t *err = reinterpret_cast<uint32_t *>(dev);
  e = cudaMemsetAsync(err, 0, sizeof(uint32_t), s->copy_in);
  io.error_word = err;
  dev += 256;
  char *at[6];
  for (size_t j = 0, off = 0; j < 6; ++j) {
    at[j] = per[j] ? dev + off : nullptr;
    off += align_up(per[j] * n, 256);
  }
  const void *ins[2] = {ids, points};
  void *outs[4] = {distance, closest, prim, geom};
  const size_t chunk = std::max<size_t>(size_t(1) << 18, (n + kHostChunks - 1) / kHostChunks);
  const size_t nchunks = (n + chunk - 1) / chunk;
  for (size_t c = 0; c < nchunks && e == cudaSuccess; ++c) {
    const size_t a = c * chunk, m = std::min(n, a + chunk) - a;
    for (int j = 0; j < 2 && e == cudaSuccess; ++j)
      if (at[j])
        e = cudaMemcpyAsync(at[j] + per[j] * a, static_cast<const char *>(ins[j]) + per[j] * a,
                            per[j] * m, cudaMemcpyHostToDevice, s->copy_in);
    cudaStream_t ks = s->streams[c % kStreams];
    if (e == cudaSuccess) e = cudaEventRecord(s->ev_in[c], s->copy_in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ks, s->ev_in[c], 0);
    bzr::DistanceIO ci = io;
    ci.n = m;
    ci.ids = at[0] ? reinterpret_cast<const uint32_t *>(at[0]) + a : nullptr;
    ci.points = reinterpret_cast<const double *>(at[1]) + 3 * a;
    ci.distance = reinterpret_cast<double *>(at[2]) + a;
    ci.closest = at[3] ? reinterpret_cast<double *>(at[3]) + 3 * a : nullptr;
    ci.prim = at[4] ? reinterpret_cast<uint32_t *>(at[4]) + a : nullptr;
    ci.geom = at[5] ? reinterpret_cast<uint32_t *>(at[5]) + a : nullptr;
    if (e == cudaSuccess)
      e = kind >= 0 ? bzr::launch_distance(s->view, kind, ci, s->plan.sms, ks)
                    : bzr::launch_nearest(s->view, ci, s->plan.sms, s->plan.pool, ks);
    if (e == cudaSuccess) e = cudaEventRecord(s->ev_done[c], ks);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->copy_out, s->ev_done[c], 0);
    for (int j = 0; j < 4 && e == cudaSuccess; ++j)
      if (outs[j])
        e = cudaMemcpyAsync(static_cast<char *>(outs[j]) + per[2 + j] * a,
                            at[2 + j] + per[2 + j] * a, per[2 + j] * m, cudaMemcpyDeviceToHost,
                            s->copy_out);
  }
  // copy_out is ordered after every chunk's kernel, and each kernel after its copies in
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->pinned_err, err, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                        s->copy_out);
  if (e != cudaSuccess) {
    // a chunk may have been left half submitted: nothing may still use the staging when it
    // goes back to the pool
    for (cudaStream_t q : {s->copy_in, s->streams[0], s->streams[1], s->streams[2], s->copy_out})
      wait_stream(q, default_timeout_ms());
    cudaFreeAsync(dev - 256, s->copy_out);
    return cuda_fail(e, "distance staging");
  }
  cudaFreeAsync(dev - 256, s->copy_out);
  (void)st;
  const int rc = staged_wait_result(s, wait_stream_spin(s->copy_out, 200));
  if (rc) return rc;
  if (s->pinned_err[0] & bzr::kErrPrimIndex)
    return fail(BZR_EINVAL, "primitive id outside the kind (its distance is NaN)");
  return BZR_OK;
}

int bzr_distance_to_surface(const bzr_scene *s, int kind, size_t n, const uint32_t *prim_ids,
                            const double *points, double *distance, double *closest,
                            void *stream) {
  if (kind < 0) return fail(BZR_EINVAL, "bad primitive kind");
  return run_distance(s, kind, n, prim_ids, points, distance, closest, nullptr, nullptr, stream);
}

int bzr_closest_surface(const bzr_scene *s, size_t n, const double *points, double *distance,
                        uint32_t *prim, uint32_t *geom, void *stream) {
  return run_distance(s, -1, n, nullptr, points, distance, nullptr, prim, geom, stream);
}

// The committed scene's bytes in the persistent format, or a negative status.
static int encode_committed(const bzr_scene *s, bzr::RawVector<uint8_t> *out) {
  if (!s) return fail(BZR_EINVAL, "scene is null");
  if (!s->host.committed) return fail(BZR_ESTATE, "scene is not committed");
  try {
    *out = bzr::encode_scene(s->host);
  } catch (const std::bad_alloc &) {
    return fail(BZR_ENOMEM, "host allocation failed while writing the scene");
  }
  return BZR_OK;
}

long bzr_scene_serialize(const bzr_scene *s, uint8_t *buffer, size_t capacity) {
  bzr::RawVector<uint8_t> b;
  const int rc = encode_committed(s, &b);
  if (rc != BZR_OK) return rc;
  if (buffer) {
    if (capacity < b.size()) return fail(BZR_EINVAL, "buffer too small for the scene");
    std::memcpy(buffer, b.data(), b.size());
  }
  return static_cast<long>(b.size());
}

int bzr_scene_deserialize(bzr_scene **out, const uint8_t *buffer, size_t size) {
  if (!out || !buffer) return fail(BZR_EINVAL, "null argument");
  *out = nullptr;
  auto *s = new (std::nothrow) bzr_scene();
  if (!s) return fail(BZR_ENOMEM, "host allocation failed");
  std::string why;
  try {
    why = bzr::decode_scene(buffer, size, &s->host);
  } catch (const std::bad_alloc &) {
    why = "host allocation failed while reading the scene";
  }
  if (!why.empty()) {
    delete s;
    return fail(BZR_EINVAL, "scene data refused: " + why);
  }
  const int rc = commit_scene(s, 0u, true);
  if (rc != BZR_OK) {
    delete s;
    return rc;
  }
  *out = s;
  return BZR_OK;
}

int bzr_scene_save(const bzr_scene *s, const char *path) {
  if (!path) return fail(BZR_EINVAL, "path is null");
  bzr::RawVector<uint8_t> b;
  const int rc = encode_committed(s, &b);
  if (rc != BZR_OK) return rc;
  std::FILE *f = std::fopen(path, "wb");
  if (!f) return fail(BZR_EINVAL, std::string("cannot open for writing: ") + path);
  const bool ok = std::fwrite(b.data(), 1, b.size(), f) == b.size();
  const bool closed = std::fclose(f) == 0;
  if (!ok || !closed) return fail(BZR_EINVAL, std::string("write failed: ") + path);
  return BZR_OK;
}

int bzr_scene_load(bzr_scene **out, const char *path) {
  if (!out || !path) return fail(BZR_EINVAL, "null argument");
  *out = nullptr;
  std::FILE *f = std::fopen(path, "rb");
  if (!f) return fail(BZR_EINVAL, std::string("cannot open: ") + path);
  bzr::RawVector<uint8_t> b;
  bool err = false;
  try {
    // One read of the size the file reports, then 64 KiB pieces up to the end of the file:
    // a pipe reports no size, procfs-like files report 0 for content they have, and a file
    // that grew after the size was taken is read to its end.
    long size = -1;
    if (std::fseek(f, 0, SEEK_END) == 0) {
      size = std::ftell(f);
      err = std::fseek(f, 0, SEEK_SET) != 0;
    }
    if (size > 0 && !err) {
      b.resize(static_cast<size_t>(size));
      const size_t got = std::fread(b.data(), 1, b.size(), f);
      b.resize(got);  // a file that shrank meanwhile: keep what was read
    }
    if (!err && !std::ferror(f)) {
      uint8_t chunk[1 << 16];
      size_t got;
      while ((got = std::fread(chunk, 1, sizeof chunk, f)) > 0)
        b.insert(b.end(), chunk, chunk + got);
    }
    err = err || std::ferror(f) != 0;
  } catch (const std::bad_alloc &) {
    std::fclose(f);
    return fail(BZR_ENOMEM, std::string("host allocation failed while reading: ") + path);
  }
  std::fclose(f);
  if (err) return fail(BZR_EINVAL, std::string("read failed: ") + path);
  if (b.empty()) return fail(BZR_EINVAL, std::string("not a scene file (empty): ") + path);
  return bzr_scene_deserialize(out, b.data(), b.size());
}

int bzr_obj_load(const char *path, double **vertices, size_t *n_vertices, uint32_t **faces,
                 size_t *n_faces) {
  if (!path || !vertices || !n_vertices || !faces || !n_faces)
    return fail(BZR_EINVAL, "null argument");
  *vertices = nullptr;
  *faces = nullptr;
  *n_vertices = *n_faces = 0;
  std::vector<double> v;
  std::vector<uint32_t> f;
  std::string why;
  try {
    why = bzr::load_obj(path, &v, &f);
  } catch (const std::bad_alloc &) {
    return fail(BZR_ENOMEM, "host allocation failed while reading the OBJ file");
  }
  if (!why.empty()) return fail(BZR_EINVAL, why);
  auto *pv = static_cast<double *>(std::malloc(std::max<size_t>(1, v.size()) * sizeof(double)));
  auto *pf = static_cast<uint32_t *>(std::malloc(std::max<size_t>(1, f.size()) * sizeof(uint32_t)));
  if (!pv || !pf) {
    std::free(pv);
    std::free(pf);
    return fail(BZR_ENOMEM, "host allocation failed");
  }
  if (!v.empty()) std::memcpy(pv, v.data(), v.size() * sizeof(double));
  if (!f.empty()) std::memcpy(pf, f.data(), f.size() * sizeof(uint32_t));
  *vertices = pv;
  *faces = pf;
  *n_vertices = v.size() / 3;
  *n_faces = f.size() / 3;
  return BZR_OK;
}

void bzr_obj_free(void *p) { std::free(p); }

int bzr_intersect1(const bzr_scene *s, const double origin[3], const double direction[3],
                   double tmin, double tmax, bzr_rayhit *rayhit, int *hit) {
  return bzr_intersect1_ex(s, origin, direction, tmin, tmax, 0u, rayhit, hit);
}

int bzr_intersect1_ex(const bzr_scene *s, const double origin[3], const double direction[3],
                      double tmin, double tmax, uint32_t ray_flags, bzr_rayhit *rayhit, int *hit) {
  if (!origin || !direction || !rayhit) return fail(BZR_EINVAL, "null argument");
  uint8_t h = 0;
  const int rc = bzr_intersectN_ex(s, 1, origin, direction, &tmin, &tmax, &rayhit->hit_distance,
                                   rayhit->uv, rayhit->normal, &rayhit->prim_id,
                                   &rayhit->geom_id, &h, BZR_MODE_FP64, ray_flags, nullptr);
  if (hit) *hit = h;
  return rc;
}

int bzr_scene_check(const bzr_scene *s, void *stream, int timeout_ms, uint32_t *flags) {
  if (!s) return fail(BZR_EINVAL, "scene is null");
  if (flags) *flags = 0;
  if (!s->host.committed) return BZR_OK;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(s->device);
  int rc = wait_stream(static_cast<cudaStream_t>(stream), timeout_ms);
  uint32_t word = 0;
  if (rc == BZR_OK) {
    const cudaError_t e =
        cudaMemcpy(&word, s->slots + kStickyWord, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = cuda_fail(e, "error word read");
  }
  cudaSetDevice(cur);
  if (rc) return rc;
  if (flags) *flags = word;
  return word ? fail(BZR_EDEVICE_FLAG, "kernel bounds check fired") : BZR_OK;
}

int bzr_scene_tune(bzr_scene *s, int option, int64_t value) {
  if (!s) return fail(BZR_EINVAL, "scene is null");
  if (!s->host.committed) return fail(BZR_ESTATE, "tune after commit");
  switch (option) {
    case BZR_TUNE_SORT:
      if (value != 0 && value != 1) return fail(BZR_EINVAL, "sort must be 0 or 1");
      s->plan.sort.enabled = value == 1 && s->sort_possible;
      return BZR_OK;
    case BZR_TUNE_SORT_MIN_RAYS:
      if (value < 0 || value > 0x7FFFFFFF) return fail(BZR_EINVAL, "bad sort threshold");
      s->plan.sort_min_rays = static_cast<uint32_t>(value);
      return BZR_OK;
    case BZR_TUNE_HOST_CHUNKS: {
      if (value < 1 || value > static_cast<int64_t>(kMaxHostChunks))
        return fail(BZR_EINVAL, "host-array chunks must be 1 to 32");
      std::lock_guard<std::mutex> lock(s->stage_mu);
      s->host_chunks = static_cast<size_t>(value);
      return BZR_OK;
    }
    case BZR_TUNE_HOST_GRID_DIV: {
      if (value < 1 || value > 8) return fail(BZR_EINVAL, "grid divisor must be 1 to 8");
      std::lock_guard<std::mutex> lock(s->stage_mu);
      s->host_grid_div = static_cast<int>(value);
      return BZR_OK;
    }
    case BZR_TUNE_HOST_EDGE: {
      if (value < 0 || value > 0x7FFFFFFF) return fail(BZR_EINVAL, "bad edge chunk size");
      std::lock_guard<std::mutex> lock(s->stage_mu);
      s->host_edge = static_cast<size_t>(value);
      return BZR_OK;
    }
    case BZR_TUNE_HOST_MIN_CHUNK: {
      if (value < 1024 || value > 0x7FFFFFFF)
        return fail(BZR_EINVAL, "host-array chunk size must be 1024 to 2^31 - 1 rays");
      std::lock_guard<std::mutex> lock(s->stage_mu);
      s->host_min_chunk = static_cast<size_t>(value);
      return BZR_OK;
    }
    case BZR_TUNE_CHUNK:
      if (value != 0 && value != 32 && value != 64 && value != 128)
        return fail(BZR_EINVAL, "rays per warp fetch must be 0 (the idle lanes), 32, 64 or 128");
      s->plan.chunk = static_cast<uint32_t>(value);
      return BZR_OK;
    case BZR_TUNE_BLOCK:
    case BZR_TUNE_STACK:
    case BZR_TUNE_TOP_NODES: {
      bzr::LaunchPlan p = s->plan;
      if (option == BZR_TUNE_BLOCK) {
        if (value != 64 && value != 128 && value != 256)
          return fail(BZR_EINVAL, "threads per block must be 64, 128 or 256");
        p.threads = static_cast<int>(value);
      } else if (option == BZR_TUNE_TOP_NODES) {
        if (value < 0 || value > 256) return fail(BZR_EINVAL, "top nodes must be 0 to 256");
        p.top_nodes = static_cast<uint32_t>(value);
      } else {
        if (value != 0 && value != 1) return fail(BZR_EINVAL, "stack storage must be 0 or 1");
        p.shared_stack = value == 1;
      }
      const bool local = !p.shared_stack && s->view.stack_cap <= bzr::kLocalStack;
      if (bzr::trace_kind_smem(s->view.stack_cap, p.threads, local, p.top_nodes) > 227 * 1024)
        return fail(BZR_EINVAL,
                    "the traversal stack and staged nodes do not fit shared memory at this "
                    "block size");
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(s->device);
      const cudaError_t e = bzr::trace_prepare(s->view, &p);
      cudaSetDevice(cur);
      if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
      s->plan = p;
      return BZR_OK;
    }
  }
  return fail(BZR_EINVAL, "unknown tuning option");
}

long bzr_scene_tree(const bzr_scene *s, int kind, double *bmin, double *bmax, uint32_t *leaf,
                    uint32_t *axis, uint32_t *children, uint32_t *prim_cnt, uint32_t *prim_ids,
                    long prim_cap) {
  if (!s || kind < 0 || kind >= bzr::kNumKinds) return fail(BZR_EINVAL, "bad argument");
  if (!s->host.committed) return fail(BZR_ESTATE, "scene is not committed");
  const bzr::Collection &c = s->host.kind[kind];
  if (!c.present) return fail(BZR_EINVAL, "kind not in the scene");
  const bzr::Tree &t = c.tree;
  const long n = static_cast<long>(t.nodes.size());
  if (!bmin || !bmax || !leaf || !axis || !children || !prim_cnt) return n;
  for (long i = 0; i < n; ++i) {
    const bzr::TreeNode &nd = t.nodes[i];
    std::memcpy(bmin + 3 * i, nd.mn, sizeof nd.mn);
    std::memcpy(bmax + 3 * i, nd.mx, sizeof nd.mx);
    leaf[i] = nd.leaf;
    axis[i] = nd.axis;
    children[2 * i] = nd.child[0];
    children[2 * i + 1] = nd.child[1];
    prim_cnt[i] = nd.leaf == 1 ? nd.prim_cnt : 0;
  }
  if (prim_ids)
    for (long i = 0; i < static_cast<long>(t.leaf_prims.size()) && i < prim_cap; ++i)
      prim_ids[i] = t.leaf_prims[i];
  return n;
}

int bzr_scene_build_statistics(const bzr_scene *s, int kind, bzr_build_statistics *out) {
  if (!s || !out) return fail(BZR_EINVAL, "null argument");
  if (kind < 0 || kind >= bzr::kNumKinds) return fail(BZR_EINVAL, "bad primitive kind");
  if (!s->host.committed) return fail(BZR_ESTATE, "scene is not committed");
  const bzr::Collection &c = s->host.kind[kind];
  if (!c.present) return fail(BZR_EINVAL, "the scene has no primitives of this kind");
  const bzr::BuildStatistics st = bzr::tree_statistics(c.tree);
  out->max_tree_depth = st.max_tree_depth;
  out->leaf_nodes = st.leaf_nodes;
  out->max_num_prims_per_leaf = st.max_num_prims_per_leaf;
  out->min_num_prims_per_leaf = st.min_num_prims_per_leaf;
  out->branch_nodes = st.branch_nodes;
  out->bad_splits = st.bad_splits;
  out->build_seconds = c.tree.build_seconds;
  return BZR_OK;
}

int bzr_scene_stats(const bzr_scene *s, int kind, uint64_t *n_nodes, uint32_t *max_depth,
                    double *build_seconds) {
  if (!s || kind < 0 || kind >= bzr::kNumKinds) return fail(BZR_EINVAL, "bad argument");
  const bzr::Collection &c = s->host.kind[kind];
  if (n_nodes) *n_nodes = c.tree.nodes.size();
  if (max_depth) *max_depth = c.tree.max_depth;
  if (build_seconds) *build_seconds = c.tree.build_seconds;
  return BZR_OK;
}

}  // extern "C"

namespace bzr {
bool injected_allocation_failure() {
  int64_t left = g_alloc_countdown.load();
  while (left > 0) {
    if (g_alloc_countdown.compare_exchange_weak(left, left - 1)) return left == 1;
  }
  return false;
}
}  // namespace bzr

int bzr_debug_fail_allocation(int64_t k) {
  if (k < 0) return fail(BZR_EINVAL, "k must be >= 0");
  g_alloc_countdown.store(k);
  return BZR_OK;
}
