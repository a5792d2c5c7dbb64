// Closest-hit traversal kernels for sm_100a.
//
// A batch runs as one persistent kernel per primitive kind present, in the reference's fixed
// order (triangles, spheres, planes, cylinders; blazert/scene.h:161-210).  Each pass merges its
// hits into the output record with the reference's rule (finalize_kind), so the result equals
// intersect1's.  Splitting by kind keeps each kernel small (registers, instruction cache) and
// keeps one kind's nodes and primitives hot in L1/L2 at a time.
//
// Work distribution: each warp owns a pool of ray indices taken from a global counter in
// chunks of kChunk (one atomic per chunk).  A lane whose ray finishes takes the next index of
// its warp's pool at once, so lanes do not idle until the slowest ray of a fixed group of 32
// is done.  Within a ray the traversal alternates "walk internal nodes to the next leaf" and
// "test the leaf's primitives", so the lanes of a warp run their leaf tests together.
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

#include "alloc.h"
#include "layout.h"
#include "bucket_sort.cuh"
#include "trace.h"
#include "trace_core.cuh"

namespace bzr {
static_assert(kSortBuckets == (size_t(1) << kSortBits), "batch sort scratch size");
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

// Shared memory of the stack: none for a thread-local stack, else stack_cap entries of 12 bytes
// per thread, rounded up to 16 bytes (the staged top-level nodes follow).
template <bool LOCAL>
__device__ __forceinline__ size_t stack_smem_bytes(uint32_t stack_cap) {
  return LOCAL ? 0 : (size_t(stack_cap) * blockDim.x * 12 + 15) / 16 * 16;
}

// Traversal stack storage.  LOCAL: a thread-local array of kLocalStack entries (local memory,
// cached in L1; the host picks it when the tree's stack fits, and it leaves the SM's shared
// memory to L1 and the occupancy to the register count).  Otherwise shared memory sized from
// the tree, entry j of thread t at [j * blockDim.x + t].  The capacity is clamped to the
// storage, so a mismatch is reported as kErrStack, never written past.
template <bool LOCAL, uint32_t LCAP = kLocalStack>
__device__ __forceinline__ void init_stack(Stack &sk, uint32_t &tid, uint32_t cap,
                                           unsigned char *smem, double *lkey, uint32_t *lref) {
  if (LOCAL) {
    sk.stride = 1;
    sk.cap = cap < LCAP ? cap : LCAP;
    sk.key = lkey;
    sk.ref = lref;
    tid = 0;
  } else {
    sk.stride = blockDim.x;
    sk.cap = cap;
    sk.key = reinterpret_cast<double *>(smem);
    sk.ref = reinterpret_cast<uint32_t *>(sk.key + size_t(sk.cap) * sk.stride);
    tid = threadIdx.x;
  }
}

// Cold start: between batches the scene may have left L2 (other work, or the benchmark's L2
// flush), and then every dependent node fetch of the first rays waits for DRAM.  The grid
// first asks L2 for the breadth-first prefix of the node array (the top levels every ray
// visits) and for the leaf-ordered primitive data, at most kPrefetchBytes of each, one
// 128-byte line per thread per round.  A hint only: nothing waits for it.
constexpr size_t kPrefetchBytes = size_t(4) << 20;

__device__ __forceinline__ void prefetch_l2(const void *base, size_t bytes) {
  if (!base) return;
  bytes = bytes < kPrefetchBytes ? bytes : kPrefetchBytes;
  const size_t step = size_t(gridDim.x) * blockDim.x * 128;
  for (size_t off = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) * 128; off < bytes;
       off += step)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(static_cast<const char *>(base) + off));
}

template <int KIND, bool MIXED>
__device__ __forceinline__ void prefetch_kind(const KindView &K) {
  if (MIXED && K.mixed_ok) {  // the wide image: nodes, then leaf records (and vertices)
    prefetch_l2(K.wide, size_t(K.n_wide) * kWideBytes);
    prefetch_l2(K.leaves, size_t(K.n_leaf16) * 16);
    if (KIND == kMesh) prefetch_l2(K.verts, size_t(K.n_verts) * kVertexDoubles * sizeof(double));
    return;
  }
  prefetch_l2(K.nodes64, size_t(K.n_internal) * kNode64Doubles * sizeof(double));
  if (KIND == kMesh) {
    prefetch_l2(K.tri, size_t(K.n_prims) * 4 * sizeof(uint32_t));
    prefetch_l2(K.verts, size_t(K.n_verts) * kVertexDoubles * sizeof(double));
  } else {
    constexpr int kDoubles = KIND == kSpheres ? 4 : KIND == kPlanes ? 14 : 16;
    prefetch_l2(K.payload, size_t(K.n_prims) * kDoubles * sizeof(double));
    prefetch_l2(K.prim_ids, size_t(K.n_prims) * sizeof(uint32_t));
  }
}

// Programmatic dependent launch (sm_90 and later): a kernel launched with programmatic stream
// serialisation may start while the kernel before it on the stream still runs, once every
// block of that kernel has called griddep_launch_dependents (or exited); griddep_wait blocks
// until that kernel has completed and its writes are visible.  Both are no-ops for a kernel
// launched without the attribute.
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void griddep_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// One kind over the whole batch.  first: this pass writes the whole output record.
// COUNT: also sums the work counters into totals[16] (per kind: box tests, primitive tests,
// node fetches, leaf fetches; see Counts).  MIXED: the rays the FP32 test covers walk the wide
// image; the others are appended to io.defer for the FP64 pass that follows (cylinders always
// take the FP64 traversal).  Keeping the FP64 walk out of the wide kernel keeps its registers
// for the wide walk.  io.n_dev: the FP64 pass over a deferred list reads its ray count there.
template <int KIND, bool COUNT, bool MIXED, bool LOCAL>
__device__ __forceinline__ void trace_kind_body(const SceneView &S, const RayIO &io, int first,
                                                uint32_t *work_counter,
                                                unsigned long long *totals) {
  constexpr bool kWide = MIXED && KIND != kCylinders;
  // The next kernel on the stream may be scheduled now: it waits (griddep_wait) for this grid
  // to complete before it reads anything this grid writes.
  griddep_launch_dependents();
  extern __shared__ __align__(16) unsigned char smem[];
  double lkey[LOCAL ? kLocalStack : 1];
  uint32_t lref[LOCAL ? kLocalStack : 1];
  Stack sk;
  uint32_t tid;
  init_stack<LOCAL>(sk, tid, S.stack_cap, smem, lkey, lref);
  const KindView &K = S.k[KIND];
  // (a deferred list is short: its pass leaves L2 to the rays)
  if (!COUNT && !io.n_dev) prefetch_kind<KIND, kWide>(K);
  // The first io.top_nodes nodes of the array this kernel walks (the top levels every ray
  // visits) are staged in shared memory after the stack.
  {
    const uint32_t avail = kWide ? K.n_wide : K.n_internal;
    const uint32_t n_top = io.top_nodes < avail ? io.top_nodes : avail;
    uint4 *top = reinterpret_cast<uint4 *>(smem + stack_smem_bytes<LOCAL>(S.stack_cap));
    const uint4 *src = kWide ? reinterpret_cast<const uint4 *>(K.wide)
                             : reinterpret_cast<const uint4 *>(K.nodes64);
    for (uint32_t j = threadIdx.x; j < n_top * 8; j += blockDim.x) top[j] = ldg(src + j);
    if (n_top) __syncthreads();
    sk.top = top;
    sk.n_top = n_top;
  }
  // Up to here only the scene was read; the counters, the rays' closest distances and the
  // deferred list come from earlier kernels of the stream.
  griddep_wait();
  const uint32_t n = io.n_dev ? *io.n_dev : io.n;
  if (n == 0) return;  // the same for every thread of the grid
  const unsigned lane = threadIdx.x & 31u;
  const unsigned below = (1u << lane) - 1u;
  uint32_t pool_next = 0, pool_end = 0;  // warp-uniform
  bool exhausted = false;                // warp-uniform
  bool active = false;
  uint32_t i = 0;
  Ray r;
  RayW f;
  float hl = 0.0f;
  KState st;
  Trav tv;
  Counts cnt = {};
  for (;;) {
    for (;;) {  // refill the idle lanes; repeats only after a lane handed its ray on
      const unsigned idle = __ballot_sync(kFull, !active);
      bool deferred = false;
      if (idle && !exhausted) {
        const uint32_t want = __popc(idle), avail = pool_end - pool_next;
        // rays taken per fetch: io.chunk (>= 32, so one fetch serves every idle lane), or
        // with io.chunk == 0 exactly the number of idle lanes the pool cannot serve
        const uint32_t take = io.chunk ? io.chunk : want - avail;
        uint32_t base = 0;
        if (want > avail) {
          if (lane == 0) base = atomicAdd(work_counter, take);
          base = __shfl_sync(kFull, base, 0);
        }
        if (!active) {
          const uint32_t rank = __popc(idle & below);
          const uint32_t idx = rank < avail ? pool_next + rank : base + (rank - avail);
          if (idx < n) {
            i = io.perm ? io.perm[idx] : idx;
            active = true;
            r = make_ray(io.org + 3 * size_t(i), io.dir + 3 * size_t(i),
                         io.tmin ? io.tmin[i] : 0.0, io.tmax ? io.tmax[i] : kDblMax);
            r.any_hit = io.any_hit != 0;
            if constexpr (kWide) {
              f = make_ray_w(r);
              if (K.mixed_ok && f.ok) {
                wtrav_begin<KIND, COUNT>(K, r, f, st, hl, tv, &cnt);
              } else {
                io.defer[atomicAdd(io.defer_count, 1u)] = i;
                active = false;
                deferred = true;
              }
            } else {
              trav_begin<KIND, COUNT>(K, r, st, tv, &cnt);
            }
          }
        }
        if (want > avail) {
          pool_next = base + (want - avail);
          pool_end = base + take;
          if (base >= n) exhausted = true;
        } else {
          pool_next += want;
        }
      }
      if (!kWide || !__any_sync(kFull, deferred)) break;
    }
    // every lane idle: the global counter has passed the end of the batch
    if (!__any_sync(kFull, active)) break;
    if (active) {
      if constexpr (kWide) {
        if (tv.live) wtrav_to_leaf<KIND, COUNT>(K, f, hl, tv, sk, tid, io.error_word, &cnt);
        while (tv.live && tv.post != kNoLeaf)
          wtrav_leaf<KIND, COUNT>(K, r, f, st, hl, tv, sk, tid, io.error_word, &cnt);
      } else {
        if (tv.live) trav_to_leaf<KIND, COUNT>(K, r, st, tv, sk, tid, io.error_word, &cnt);
        if (tv.live) trav_leaf<KIND, COUNT>(K, r, st, tv, sk, tid, io.error_word, &cnt);
      }
      if (!tv.live) {
        if constexpr (kWide) wtrav_end<KIND>(K, r, st);
        finalize_kind<KIND>(S, r, st, i, first != 0, io.t, io.uv, io.normal, io.prim, io.geom,
                            io.hit);
        active = false;
      }
    }
  }
  if (COUNT) {
    for (int k = 0; k < kNumKinds; ++k) {
      unsigned long long v[4] = {cnt.box[k], cnt.prim[k], cnt.node[k], cnt.leaf[k]};
      for (int j = 0; j < 4; ++j) {
        for (int off = 16; off > 0; off >>= 1) v[j] += __shfl_down_sync(kFull, v[j], off);
        if (lane == 0 && v[j]) atomicAdd(totals + j * kNumKinds + k, v[j]);
      }
    }
  }
}

// The FP64 kernels, and the mixed-precision kernels with a register cap: the wide walk keeps
// the FP64 ray and hit state live beside its FP32 node state, and its latency-bound loop gains
// more from resident warps than it loses to the cap.
template <int KIND, bool COUNT, bool LOCAL>
__global__ void __launch_bounds__(kMaxTraceThreads)
    trace_kind_kernel(SceneView S, RayIO io, int first, uint32_t *work_counter,
                      unsigned long long *totals) {
  trace_kind_body<KIND, COUNT, false, LOCAL>(S, io, first, work_counter, totals);
}

#ifndef BZR_WIDE_REGS
#define BZR_WIDE_REGS 72
#endif
template <int KIND, bool COUNT, bool LOCAL>
__global__ void __maxnreg__(BZR_WIDE_REGS)
    trace_wide_kernel(SceneView S, RayIO io, int first, uint32_t *work_counter,
                      unsigned long long *totals) {
  trace_kind_body<KIND, COUNT, true, LOCAL>(S, io, first, work_counter, totals);
}

template <int KIND, bool COUNT, bool MIXED, bool LOCAL>
constexpr auto trace_kernel() {
  if constexpr (MIXED)
    return trace_wide_kernel<KIND, COUNT, LOCAL>;
  else
    return trace_kind_kernel<KIND, COUNT, LOCAL>;
}

// Batching form: one kind over many scenes.  Warps take chunks of one scene's rays; a lane
// keeps its own ray's scene, so a warp may finish rays of one scene while starting another's.
// The pass of a scene's first kind writes its whole record; the pass of its last kind
// completes it and stamps the scene's completion time.
// LCAP: entries of the thread-local stack (the batch's stack-depth knob: 32 or 64).
template <int KIND, bool MIXED, bool LOCAL, uint32_t LCAP>
__device__ __forceinline__ void trace_batch_body(const BatchView &B, const RayIO &io,
                                                 uint32_t *chunk_counter, uint32_t stack_cap) {
  constexpr bool kWide = MIXED && KIND != kCylinders;
  extern __shared__ __align__(16) unsigned char smem[];
  double lkey[LOCAL ? LCAP : 1];
  uint32_t lref[LOCAL ? LCAP : 1];
  Stack sk;
  uint32_t tid;
  init_stack<LOCAL, LCAP>(sk, tid, stack_cap, smem, lkey, lref);
  const unsigned lane = threadIdx.x & 31u;
  const unsigned below = (1u << lane) - 1u;
  uint32_t pool_next = 0, pool_end = 0, pool_scene = 0;  // warp-uniform
  bool exhausted = false;
  bool active = false;
  uint32_t i = 0, sc = 0;
  const KindView *K = nullptr;
  Ray r;
  RayW f;
  float hl = 0.0f;
  bool use32 = false;
  KState st;
  Trav tv;
  Counts cnt = {};
  for (;;) {
    const unsigned idle = __ballot_sync(kFull, !active);
    if (idle && !exhausted) {
      const uint32_t want = __popc(idle), avail = pool_end - pool_next;
      const uint32_t rank = __popc(idle & below);
      uint32_t base = 0, cbegin = 0, cend = 0, cscene = 0;
      bool got_chunk = false;
      if (want > avail) {  // next chunk that has this kind
        uint32_t c = 0;
        for (;;) {
          if (lane == 0) c = atomicAdd(chunk_counter, 1u);
          c = __shfl_sync(kFull, c, 0);
          if (c >= B.n_chunks) {
            exhausted = true;
            break;
          }
          const BatchChunk ch = B.chunks[c];
          if (B.views[ch.scene].k[KIND].present && B.views[ch.scene].k[KIND].n_prims) {
            cbegin = ch.begin;
            cend = ch.end;
            cscene = ch.scene;
            got_chunk = true;
            break;
          }
        }
        base = cbegin;
      }
      if (!active) {
        uint32_t idx = 0, s2 = 0;
        bool ok = false;
        if (rank < avail) {
          idx = pool_next + rank;
          s2 = pool_scene;
          ok = true;
        } else if (got_chunk && base + (rank - avail) < cend) {
          idx = base + (rank - avail);
          s2 = cscene;
          ok = true;
        }
        if (ok) {
          i = io.perm ? io.perm[idx] : idx;  // a sorted batch keeps each scene's range
          sc = s2;
          active = true;
          K = &B.views[sc].k[KIND];
          r = make_ray(io.org + 3 * size_t(i), io.dir + 3 * size_t(i), io.tmin ? io.tmin[i] : 0.0,
                       io.tmax ? io.tmax[i] : kDblMax);
          r.any_hit = io.any_hit != 0;
          if constexpr (kWide) {
            f = make_ray_w(r);
            use32 = K->mixed_ok && f.ok;
          }
          if (kWide && use32)
            wtrav_begin<KIND, false>(*K, r, f, st, hl, tv, &cnt);
          else
            trav_begin<KIND, false>(*K, r, st, tv, &cnt);
        }
      }
      if (want > avail) {
        if (got_chunk) {
          const uint32_t used = want - avail;
          pool_next = cbegin + (used < cend - cbegin ? used : cend - cbegin);
          pool_end = cend;
          pool_scene = cscene;
        } else {
          pool_next = pool_end;
        }
      } else {
        pool_next += want;
      }
    }
    if (!__any_sync(kFull, active)) break;
    if (active) {
      if (kWide && use32) {
        if (tv.live) wtrav_to_leaf<KIND, false>(*K, f, hl, tv, sk, tid, io.error_word, &cnt);
        while (tv.live && tv.post != kNoLeaf)
          wtrav_leaf<KIND, false>(*K, r, f, st, hl, tv, sk, tid, io.error_word, &cnt);
      } else {
        if (tv.live) trav_to_leaf<KIND, false>(*K, r, st, tv, sk, tid, io.error_word, &cnt);
        if (tv.live) trav_leaf<KIND, false>(*K, r, st, tv, sk, tid, io.error_word, &cnt);
      }
      if (!tv.live) {
        if (kWide && use32) wtrav_end<KIND>(*K, r, st);
        finalize_kind<KIND>(B.views[sc], r, st, i, B.first_kind[sc] == KIND, io.t, io.uv,
                            io.normal, io.prim, io.geom, io.hit);
        if (B.last_kind[sc] == KIND && B.scene_left) {
          if (atomicSub(B.scene_left + sc, 1u) == 1u && B.scene_done_ns) {
            __threadfence();
            unsigned long long now;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
            B.scene_done_ns[sc] = now;
          }
        }
        active = false;
      }
    }
  }
}

// The batch's FP64 kernels, and its mixed kernels under a register cap, as trace_wide_kernel.
// The batch's scenes are small and mostly in L2, so its walk waits less on memory: on 256
// icospheres the cap measured 1,180 (none), 1,188 (72), 1,224 (80) and 1,215 (96) Mrays/s.
#ifndef BZR_BATCH_WIDE_REGS
#define BZR_BATCH_WIDE_REGS 80
#endif
template <int KIND, bool LOCAL, uint32_t LCAP>
__global__ void __launch_bounds__(kMaxTraceThreads)
    trace_batch_kernel(BatchView B, RayIO io, uint32_t *chunk_counter, uint32_t stack_cap) {
  trace_batch_body<KIND, false, LOCAL, LCAP>(B, io, chunk_counter, stack_cap);
}
template <int KIND, bool LOCAL, uint32_t LCAP>
__global__ void __maxnreg__(BZR_BATCH_WIDE_REGS)
    trace_batch_wide_kernel(BatchView B, RayIO io, uint32_t *chunk_counter, uint32_t stack_cap) {
  trace_batch_body<KIND, true, LOCAL, LCAP>(B, io, chunk_counter, stack_cap);
}
template <int KIND, bool MIXED, bool LOCAL, uint32_t LCAP>
constexpr auto batch_fn() {
  if constexpr (MIXED)
    return trace_batch_wide_kernel<KIND, LOCAL, LCAP>;
  else
    return trace_batch_kernel<KIND, LOCAL, LCAP>;
}

__global__ void batch_start_kernel(BatchView B, uint32_t n_scenes) {
  for (uint32_t s = threadIdx.x; s < n_scenes; s += blockDim.x)
    if (B.scene_left) B.scene_left[s] = B.scene_rays[s];
  if (threadIdx.x == 0 && B.start_ns) {
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    *B.start_ns = now;
  }
}

// Output defaults for every ray of a scene without primitives (blazert/ray.h:80-84).
__global__ void fill_defaults_kernel(RayIO io) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < io.n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    if (io.t) io.t[i] = kDblMax;
    if (io.uv) io.uv[2 * i] = io.uv[2 * i + 1] = 0.0;
    if (io.normal) io.normal[3 * i] = io.normal[3 * i + 1] = io.normal[3 * i + 2] = 0.0;
    if (io.prim) io.prim[i] = 0xFFFFFFFFu;
    if (io.geom) io.geom[i] = 0xFFFFFFFFu;
    if (io.hit) io.hit[i] = 0;
  }
}

// -------------------------------------------------------------------------- coherence sort
// Sort keys of a batch of many scenes: the scene index in the top scene_bits bits, then the
// single-scene key (direction octant over the origin's Morton code in the scene's box), so
// that the counting sort keeps every scene's rays in the scene's own range.  One warp per
// chunk of the chunk table, which covers every ray of the batch when the batch is sorted
// (scenes with nothing to trace included).
__global__ void batch_sort_key_kernel(BatchView B, RayIO io, uint32_t *keys, uint32_t *counts) {
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < B.n_chunks;
       c += warps) {
    const BatchChunk ch = B.chunks[c];
    const RaySort rs = B.scene_sort[ch.scene];
    for (uint32_t p = ch.begin + lane; p < ch.end; p += 32) {
      const double *o = io.org + 3 * size_t(p), *d = io.dir + 3 * size_t(p);
      uint32_t q[3];
      for (int a = 0; a < 3; ++a) {
        float x = (float(o[a]) - rs.lo[a]) * rs.scale[a];
        x = fminf(fmaxf(x, 0.0f), 511.0f);  // NaN maps to 0
        q[a] = uint32_t(x);
      }
      const uint32_t oct = (d[0] < 0.0 ? 4u : 0u) | (d[1] < 0.0 ? 2u : 0u) | (d[2] < 0.0 ? 1u : 0u);
      const uint32_t low = (oct << 27) | (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
      const uint32_t k = B.scene_bits >= 2 ? (uint32_t(ch.scene) << (32 - B.scene_bits)) |
                                                 (low >> (B.scene_bits - 2))
                                           : (uint32_t(ch.scene) << 31) | (low << 1);
      keys[p] = k;
      atomicAdd(counts + (k >> (32 - kSortBits)), 1u);
    }
  }
}

__device__ __forceinline__ uint32_t ray_key(const RayIO &io, const RaySort &rs, uint32_t i) {
  const double *o = io.org + 3 * size_t(i), *d = io.dir + 3 * size_t(i);
  uint32_t q[3];
  for (int a = 0; a < 3; ++a) {
    float x = (float(o[a]) - rs.lo[a]) * rs.scale[a];
    x = fminf(fmaxf(x, 0.0f), 511.0f);  // NaN maps to 0
    q[a] = uint32_t(x);
  }
  const uint32_t oct = (d[0] < 0.0 ? 4u : 0u) | (d[1] < 0.0 ? 2u : 0u) | (d[2] < 0.0 ? 1u : 0u);
  return (oct << 27) | (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
}

__global__ void sort_histogram_kernel(RayIO io, RaySort rs, uint32_t *keys, uint32_t *counts) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < io.n; i += gridDim.x * blockDim.x) {
    const uint32_t k = ray_key(io, rs, i);
    keys[i] = k;
    atomicAdd(counts + (k >> (32 - kSortBits)), 1u);
  }
}

// The counting kernels (measurement only) always keep the stack in shared memory; the
// tracing kernels use the thread-local stack whenever the tree's stack fits it, unless the
// plan asks for shared memory.
inline bool use_local(const SceneView &S, const LaunchPlan &plan) {
  return !plan.shared_stack && S.stack_cap <= kLocalStack;
}

// Whether a pass of KIND in `mode` walks the wide image (and defers the rays it cannot).
template <int KIND>
bool walks_wide(const SceneView &S, int mode) {
  return mode == kModeMixed && KIND != kCylinders && S.k[KIND].present && S.k[KIND].n_prims &&
         S.k[KIND].mixed_ok;
}

using TraceFn = void (*)(SceneView, RayIO, int, uint32_t *, unsigned long long *);

// One trace kernel on `stream`; early: launched with programmatic stream serialisation (the
// kernel before it on the stream is a trace kernel of the same call; see griddep_wait).
cudaError_t launch_one(TraceFn fn, int blocks, int threads, size_t smem, cudaStream_t stream,
                       bool early, const SceneView &S, const RayIO &io, int first,
                       uint32_t *counter, unsigned long long *totals) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(blocks));
  cfg.blockDim = dim3(unsigned(threads));
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = early ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, fn, S, io, first, counter, totals);
}

// The pass of one kind: one kernel, or for a wide walk the wide kernel and then the FP64
// kernel over the rays it deferred.  counters: the kTraceCounterWords words of the call;
// after_trace: a trace kernel of this call precedes the pass on the stream.
template <int KIND, bool COUNT>
cudaError_t launch_kind(const SceneView &S, const RayIO &io, int mode, int first,
                        bool after_trace, const LaunchPlan &plan, cudaStream_t stream,
                        uint32_t *counters, unsigned long long *totals) {
  const int th = plan.threads;
  const bool local = !COUNT && use_local(S, plan);
  const size_t smem = trace_kind_smem(S.stack_cap, th, local, io.top_nodes);
  const bool early = after_trace && plan.early_launch;
  const TraceFn fp64 = local ? trace_kernel<KIND, false, false, true>()
                             : trace_kernel<KIND, COUNT, false, false>();
  if (!walks_wide<KIND>(S, mode))
    return launch_one(fp64, plan.blocks[KIND], th, smem, stream, early, S, io, first,
                      counters + KIND, totals);
  const TraceFn wide_fn = local ? trace_kernel<KIND, false, true, true>()
                                : trace_kernel<KIND, COUNT, true, false>();
  RayIO wide = io;
  wide.defer_count = counters + kNumKinds + KIND;
  RayIO rest = io;
  rest.perm = io.defer;  // ray indices
  rest.n_dev = wide.defer_count;
  const cudaError_t e = launch_one(wide_fn, plan.blocks32[KIND], th, smem, stream, early, S,
                                   wide, first, counters + KIND, totals);
  if (e != cudaSuccess) return e;
  return launch_one(fp64, plan.blocks[KIND], th, smem, stream, plan.early_launch, S, rest, first,
                    counters + 2 * kNumKinds + KIND, totals);
}

// Resident blocks per SM of `fn` with `threads` per block and `smem` bytes of dynamic shared
// memory, times the SMs.
cudaError_t grid_for(const void *fn, int threads, size_t smem, int sms, int *blocks) {
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
  if (e != cudaSuccess) return e;
  *blocks = sms * (per_sm > 0 ? per_sm : 1);
  return cudaSuccess;
}

template <int KIND>
cudaError_t prepare_kind(const SceneView &S, LaunchPlan *plan) {
  const int th = plan->threads;
  const size_t smem = trace_kind_smem(S.stack_cap, th, false, plan->top_nodes);
  const size_t smem_local = trace_kind_smem(S.stack_cap, th, true, plan->top_nodes);
  const void *shared_fns[4] = {
      reinterpret_cast<const void *>(trace_kernel<KIND, false, false, false>()),
      reinterpret_cast<const void *>(trace_kernel<KIND, true, false, false>()),
      reinterpret_cast<const void *>(trace_kernel<KIND, false, true, false>()),
      reinterpret_cast<const void *>(trace_kernel<KIND, true, true, false>())};
  int ignored = 0;
  for (const void *fn : shared_fns) {
    const cudaError_t e = grid_for(fn, th, smem, plan->sms, &ignored);
    if (e != cudaSuccess) return e;
  }
  int *blocks = &plan->blocks[KIND], *blocks32 = &plan->blocks32[KIND];
  if (use_local(S, *plan)) {
    const cudaError_t e = grid_for(
        reinterpret_cast<const void *>(trace_kernel<KIND, false, false, true>()), th,
        smem_local, plan->sms, blocks);
    if (e != cudaSuccess) return e;
    return grid_for(reinterpret_cast<const void *>(trace_kernel<KIND, false, true, true>()), th,
                    smem_local, plan->sms, blocks32);
  }
  const cudaError_t e = grid_for(shared_fns[0], th, smem, plan->sms, blocks);
  if (e != cudaSuccess) return e;
  return grid_for(shared_fns[2], th, smem, plan->sms, blocks32);
}

}  // namespace

cudaError_t launch_defaults(const RayIO &io, int sms, cudaStream_t stream) {
  const int threads = 256;
  const uint64_t want = (uint64_t(io.n) + threads - 1) / threads;
  const int blocks = int(want < uint64_t(sms) * 8 ? (want ? want : 1) : uint64_t(sms) * 8);
  fill_defaults_kernel<<<blocks, threads, 0, stream>>>(io);
  return cudaGetLastError();
}

size_t trace_smem_bytes(uint32_t stack_cap, int threads) {
  return size_t(stack_cap) * threads * (sizeof(double) + sizeof(uint32_t));
}

size_t trace_kind_smem(uint32_t stack_cap, int threads, bool local, uint32_t top_nodes) {
  const size_t stack = local ? 0 : (trace_smem_bytes(stack_cap, threads) + 15) / 16 * 16;
  return stack + size_t(top_nodes) * 128;
}

cudaError_t trace_prepare(const SceneView &S, LaunchPlan *plan) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  plan->sms = sms;
  if ((e = prepare_kind<kMesh>(S, plan)) != cudaSuccess) return e;
  if ((e = prepare_kind<kSpheres>(S, plan)) != cudaSuccess) return e;
  if ((e = prepare_kind<kPlanes>(S, plan)) != cudaSuccess) return e;
  return prepare_kind<kCylinders>(S, plan);
}

int trace_passes(const SceneView &S) {
  int n = 0;
  for (int k = 0; k < kNumKinds; ++k) n += (S.k[k].present && S.k[k].n_prims) ? 1 : 0;
  return n;
}

cudaError_t launch_trace(const SceneView &S, const RayIO &io, int mode, const LaunchPlan &plan,
                         cudaStream_t stream, uint32_t *counters, unsigned long long *totals) {
  cudaError_t e = cudaMemsetAsync(counters, 0, kTraceCounterWords * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  RayIO sorted = io;
  sorted.chunk = plan.chunk;
  sorted.top_nodes = plan.top_nodes;
  sorted.n_dev = nullptr;
  // scratch from the pool: the sort's keys, permutation and bucket counts, then the deferred
  // list of the wide passes unless the caller gave one
  const bool sort = plan.sort.enabled && io.n >= plan.sort_min_rays && trace_passes(S) > 0;
  const bool defer = !io.defer && (walks_wide<kMesh>(S, mode) || walks_wide<kSpheres>(S, mode) ||
                                   walks_wide<kPlanes>(S, mode));
  const size_t nb = size_t(1) << kSortBits;
  const size_t sort_words = sort ? 2 * size_t(io.n) + nb : 0;
  uint32_t *scratch = nullptr;
  if (sort || defer) {
    e = bzr::pool_malloc(&scratch, (sort_words + (defer ? io.n : 0)) * sizeof(uint32_t),
                         plan.pool, stream);
    if (e != cudaSuccess) return e;
    if (defer) sorted.defer = scratch + sort_words;
  }
  if (sort) {
    uint32_t *keys = scratch, *perm = scratch + io.n, *counts = scratch + 2 * size_t(io.n);
    e = cudaMemsetAsync(counts, 0, nb * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    const int blocks = plan.sms * 8;
    sort_histogram_kernel<<<blocks, 256, 0, stream>>>(io, plan.sort, keys, counts);
    bucket_scan_kernel<<<1, 1024, 0, stream>>>(counts);
    bucket_scatter_kernel<<<blocks, 256, 0, stream>>>(io.n, keys, counts, perm);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    sorted.perm = perm;
  }
  const RayIO &run = sorted;
  int first = 1;
  for (int k = 0; k < kNumKinds; ++k) {
    if (!S.k[k].present || S.k[k].n_prims == 0) continue;
    uint32_t *c = counters;
    const bool after = !first;
    switch (k) {
      case kMesh:
        e = totals ? launch_kind<kMesh, true>(S, run, mode, first, after, plan, stream, c, totals)
                   : launch_kind<kMesh, false>(S, run, mode, first, after, plan, stream, c,
                                               nullptr);
        break;
      case kSpheres:
        e = totals ? launch_kind<kSpheres, true>(S, run, mode, first, after, plan, stream, c,
                                                 totals)
                   : launch_kind<kSpheres, false>(S, run, mode, first, after, plan, stream, c,
                                                  nullptr);
        break;
      case kPlanes:
        e = totals ? launch_kind<kPlanes, true>(S, run, mode, first, after, plan, stream, c,
                                                totals)
                   : launch_kind<kPlanes, false>(S, run, mode, first, after, plan, stream, c,
                                                 nullptr);
        break;
      default:
        e = totals ? launch_kind<kCylinders, true>(S, run, mode, first, after, plan, stream, c,
                                                   totals)
                   : launch_kind<kCylinders, false>(S, run, mode, first, after, plan, stream, c,
                                                    nullptr);
        break;
    }
    if (e != cudaSuccess) break;  // the scratch is still released below
    first = 0;
  }
  if (first && e == cudaSuccess) {  // nothing to trace
    const int threads = 256;
    const uint64_t want = (uint64_t(io.n) + threads - 1) / threads;
    const int blocks = int(want < uint64_t(plan.sms) * 8 ? want : uint64_t(plan.sms) * 8);
    fill_defaults_kernel<<<blocks > 0 ? blocks : 1, threads, 0, stream>>>(io);
    e = cudaGetLastError();
  }
  if (scratch) {
    const cudaError_t f = cudaFreeAsync(scratch, stream);
    if (e == cudaSuccess) e = f;
  }
  return e;
}

namespace {
// The kernel a batch launch uses for one kind: stack storage (thread-local with 32 or 64
// entries, or shared) and mode.
template <int KIND, bool MIXED>
const void *batch_kernel(bool local, uint32_t lcap) {
  if (local && lcap == 32) return reinterpret_cast<const void *>(batch_fn<KIND, MIXED, true, 32>());
  if (local) return reinterpret_cast<const void *>(batch_fn<KIND, MIXED, true, kLocalStack>());
  return reinterpret_cast<const void *>(batch_fn<KIND, MIXED, false, kLocalStack>());
}

inline bool batch_local(uint32_t stack_cap, const BatchPlan &plan) {
  return !plan.shared_stack && stack_cap <= plan.local_stack;
}

template <int KIND>
cudaError_t prepare_batch_kind(uint32_t stack_cap, const BatchPlan &plan, int *blocks,
                               int *blocks32) {
  const int sms = plan.sms, th = plan.threads;
  const bool local = batch_local(stack_cap, plan);
  const size_t smem = local ? 0 : trace_smem_bytes(stack_cap, th);
  const cudaError_t e = grid_for(batch_kernel<KIND, false>(local, plan.local_stack), th, smem, sms,
                                 blocks);
  if (e != cudaSuccess) return e;
  return grid_for(batch_kernel<KIND, true>(local, plan.local_stack), th, smem, sms, blocks32);
}
}  // namespace

cudaError_t batch_prepare(uint32_t stack_cap, BatchPlan *plan) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  plan->sms = sms;
  plan->stack_cap = stack_cap;
  if ((e = prepare_batch_kind<kMesh>(stack_cap, *plan, &plan->blocks[kMesh],
                                     &plan->blocks32[kMesh])) != cudaSuccess)
    return e;
  if ((e = prepare_batch_kind<kSpheres>(stack_cap, *plan, &plan->blocks[kSpheres],
                                        &plan->blocks32[kSpheres])) != cudaSuccess)
    return e;
  if ((e = prepare_batch_kind<kPlanes>(stack_cap, *plan, &plan->blocks[kPlanes],
                                       &plan->blocks32[kPlanes])) != cudaSuccess)
    return e;
  return prepare_batch_kind<kCylinders>(stack_cap, *plan, &plan->blocks[kCylinders],
                                        &plan->blocks32[kCylinders]);
}

cudaError_t launch_batch(const BatchView &B, const RayIO &io, int mode, const BatchPlan &plan,
                         cudaStream_t stream, uint32_t *counters,
                         const BatchSortScratch &sort_scratch) {
  cudaError_t e = cudaMemsetAsync(counters, 0, kNumKinds * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  batch_start_kernel<<<1, 256, 0, stream>>>(B, B.n_scenes);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  RayIO run = io;
  if (plan.sort && sort_scratch.perm && B.n_chunks) {
    // every ray of the batch gets a scene-major key; rays of scenes without chunks are never
    // taken from the permutation, so their keys only need to land in their scene's range
    e = cudaMemsetAsync(sort_scratch.counts, 0, (size_t(1) << kSortBits) * sizeof(uint32_t),
                        stream);
    if (e != cudaSuccess) return e;
    const int blocks = plan.sms * 8;
    batch_sort_key_kernel<<<blocks, 256, 0, stream>>>(B, io, sort_scratch.keys,
                                                      sort_scratch.counts);
    bucket_scan_kernel<<<1, 1024, 0, stream>>>(sort_scratch.counts);
    bucket_scatter_kernel<<<blocks, 256, 0, stream>>>(io.n, sort_scratch.keys,
                                                      sort_scratch.counts, sort_scratch.perm);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    run.perm = sort_scratch.perm;
  }
  const bool local = batch_local(plan.stack_cap, plan);
  const int th = plan.threads;
  const size_t smem = local ? 0 : trace_smem_bytes(plan.stack_cap, th);
  for (int k = 0; k < kNumKinds; ++k) {
    if (!(plan.kinds_present & (1 << k))) continue;
    // cylinders, and every kind at node width 2: the FP64 traversal
    const bool m = mode == kModeMixed && k != kCylinders && plan.node_width == 8;
    const int b = m ? plan.blocks32[k] : plan.blocks[k];
    uint32_t *c = counters + k;
#define BZR_BATCH_LAUNCH(KK)                                                                   \
  if (local && plan.local_stack == 32) {                                                       \
    if (m)                                                                                     \
      batch_fn<KK, true, true, 32>()<<<b, th, 0, stream>>>(B, run, c, plan.stack_cap);          \
    else                                                                                       \
      batch_fn<KK, false, true, 32>()<<<b, th, 0, stream>>>(B, run, c, plan.stack_cap);         \
  } else if (local) {                                                                          \
    if (m)                                                                                     \
      batch_fn<KK, true, true, kLocalStack>()<<<b, th, 0, stream>>>(B, run, c, plan.stack_cap); \
    else                                                                                       \
      batch_fn<KK, false, true, kLocalStack>()<<<b, th, 0, stream>>>(B, run, c,                 \
                                                                   plan.stack_cap);            \
  } else if (m) {                                                                              \
    batch_fn<KK, true, false, kLocalStack>()<<<b, th, smem, stream>>>(B, run, c,                \
                                                                    plan.stack_cap);           \
  } else {                                                                                     \
    batch_fn<KK, false, false, kLocalStack>()<<<b, th, smem, stream>>>(B, run, c,               \
                                                                     plan.stack_cap);          \
  }
    switch (k) {
      case kMesh: BZR_BATCH_LAUNCH(kMesh); break;
      case kSpheres: BZR_BATCH_LAUNCH(kSpheres); break;
      case kPlanes: BZR_BATCH_LAUNCH(kPlanes); break;
      default: BZR_BATCH_LAUNCH(kCylinders); break;
    }
#undef BZR_BATCH_LAUNCH
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace bzr
