// GPU binned-SAH builder for sm_100a that reproduces the host builder's tree (and so the
// reference's, blazert/bvh/builder.h:84-226 with blazert/bvh/binbuffer.h:66-167) node for node.
//
// The host builder recurses depth first; every decision it takes for a node depends only on
// the node's primitive range, so the nodes of one tree level can be built at once.  One CTA
// builds one node of the current level:
//  1. the node box, a min/max reduction over its primitives' boxes;
//  2. leaf when the range holds at most min_leaf primitives or depth reached max_depth;
//  3. otherwise the 3 x bins bins of the centres (count and box per bin) in shared memory,
//     the slot computed with the host's expression and rounding;
//  4. the SAH sweep of each axis by one thread, in the host's order and arithmetic (compiled
//     with --fmad=false, like the host with -ffp-contract=off), giving best cost and cut;
//  5. the counts of centres below the cut on each axis decide the host's attempt sequence
//     (a split that puts everything on one side moves to the next axis; three such attempts
//     fall back to the middle of the range);
//  6. the partition std::partition performs (libstdc++, bidirectional iterators: the k-th
//     element failing the predicate from the left is swapped with the k-th element passing it
//     from the right), computed with block-wide prefix sums;
//  7. two child ranges for the next level.
// Leaves in DFS order take their primitives left to right from the final id array, so that
// array is the host's leaf-primitive list.  The level-order node records are renumbered into
// the host's DFS pre-order on the host.
//
// min and max commute for the finite values the builder accepts (non-finite boxes or centres
// fall back to the host builder), so the reductions give the host's boxes; only the sign of
// a zero bound can differ, which no decision and no traversal comparison can see.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "alloc.h"
#include "scene.h"

namespace bzr {
namespace {

constexpr int kThreads = 256;
constexpr double kMax = 1.7976931348623157e308;
// Ranges of at least kWidePrims primitives are built by a cluster of kCluster CTAs that share
// their partial boxes, bins and counts through distributed shared memory.
constexpr uint32_t kWidePrims = 1u << 14;
constexpr unsigned kCluster = 8;

struct Seg {
  uint32_t begin, end, depth, node;
};

struct GNode {
  double mn[3], mx[3];
  uint32_t leaf, axis, begin, end, child0, child1;
};

// Totally ordered integer image of a finite double (for shared-memory atomic min / max).
__device__ __forceinline__ long long okey(double d) {
  const long long b = __double_as_longlong(d);
  return b >= 0 ? b : b ^ 0x7FFFFFFFFFFFFFFFLL;
}
__device__ __forceinline__ double ukey(long long k) {
  return __longlong_as_double(k >= 0 ? k : k ^ 0x7FFFFFFFFFFFFFFFLL);
}

// Block-wide exclusive prefix sum of one flag per thread; returns this thread's rank and
// writes the block total to *total (every thread).
__device__ __forceinline__ uint32_t block_rank(bool flag, uint32_t *warp_sums, uint32_t *total) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned ball = __ballot_sync(0xFFFFFFFFu, flag);
  const uint32_t in_warp = __popc(ball & ((1u << lane) - 1u));
  if (lane == 0) warp_sums[warp] = __popc(ball);
  __syncthreads();
  uint32_t before = 0, all = 0;
  for (unsigned w = 0; w < blockDim.x / 32; ++w) {
    const uint32_t v = warp_sums[w];
    if (w < warp) before += v;
    all += v;
  }
  __syncthreads();
  *total = all;
  return before + in_warp;
}

__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
  return v;
}

// Surface area as blazert/bvh/binbuffer.h:16-19 computes it (the host's surface()).
__device__ __forceinline__ double surface(const double *mn, const double *mx) {
  const double e0 = fabs(mx[0] - mn[0]), e1 = fabs(mx[1] - mn[1]), e2 = fabs(mx[2] - mn[2]);
  return 2.0 * ((e0 * e1 + e1 * e2) + e2 * e0);
}

// Shared-memory bins of one node: per axis and bin 6 ordered box keys, the right-hand cost
// and the count.
struct Bins {
  long long *keys;  // 3 * nb * 6
  double *rcost;    // 3 * nb
  uint32_t *count;  // 3 * nb
};
__device__ __forceinline__ Bins bins_at(unsigned char *smem, uint32_t nb) {
  Bins b;
  b.keys = reinterpret_cast<long long *>(smem);
  b.rcost = reinterpret_cast<double *>(b.keys + 18 * size_t(nb));
  b.count = reinterpret_cast<uint32_t *>(b.rcost + 3 * size_t(nb));
  return b;
}
constexpr size_t bins_bytes(uint32_t nb) { return (8 * 18 + 8 * 3 + 4 * 3) * size_t(nb); }

__device__ void bins_clear(const Bins &B, uint32_t nb) {
  for (uint32_t i = threadIdx.x; i < 3 * nb; i += blockDim.x) {
    for (int q = 0; q < 3; ++q) {
      B.keys[6 * i + q] = okey(kMax);
      B.keys[6 * i + 3 + q] = okey(-kMax);
    }
    B.count[i] = 0;
  }
}

// Node box of positions [a, b) of ids, reduced over the block into box[6] (valid for every
// thread after the call).
__device__ void box_reduce(const double *bmin, const double *bmax, const uint32_t *ids,
                           uint32_t a, uint32_t b, double (*red)[3][kThreads / 32], double *box) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  double mn[3] = {kMax, kMax, kMax}, mx[3] = {-kMax, -kMax, -kMax};
  for (uint32_t i = a + threadIdx.x; i < b; i += blockDim.x) {
    const size_t id = ids[i];
    for (int k = 0; k < 3; ++k) {
      mn[k] = fmin(mn[k], bmin[3 * id + k]);
      mx[k] = fmax(mx[k], bmax[3 * id + k]);
    }
  }
  for (int k = 0; k < 3; ++k) {
    mn[k] = warp_min(mn[k]);
    mx[k] = warp_max(mx[k]);
    if (lane == 0) {
      red[0][k][warp] = mn[k];
      red[1][k][warp] = mx[k];
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int k = threadIdx.x;
    double lo = kMax, hi = -kMax;
    for (unsigned w = 0; w < blockDim.x / 32; ++w) {
      lo = fmin(lo, red[0][k][w]);
      hi = fmax(hi, red[1][k][w]);
    }
    box[k] = lo;
    box[3 + k] = hi;
  }
  __syncthreads();
}

// Bins the centres of positions [a, b) of ids (the node box given).
__device__ void bin_prims(const Bins &B, const double *bmin, const double *bmax,
                          const double *ctr, const uint32_t *ids, uint32_t a, uint32_t b,
                          const double *box, uint32_t nb) {
  double inv[3];
  for (int k = 0; k < 3; ++k) {
    const double ext = box[3 + k] - box[k];
    inv[k] = ext > 0.0 ? 1.0 / ext : 0.0;
  }
  for (uint32_t i = a + threadIdx.x; i < b; i += blockDim.x) {
    const size_t id = ids[i];
    for (int k = 0; k < 3; ++k) {
      const double pos = ((ctr[3 * id + k] - box[k]) * inv[k]) * static_cast<double>(nb - 1);
      // the host's min(nb - 1, unsigned(max(0u, unsigned(round(pos))))), with the
      // double -> unsigned conversion going through a 64-bit signed integer
      const unsigned r = static_cast<unsigned>(static_cast<long long>(round(pos)));
      const uint32_t slot = min(nb - 1, max(0u, r));
      const uint32_t c = k * nb + slot;
      atomicAdd(B.count + c, 1u);
      for (int q = 0; q < 3; ++q) {
        atomicMin(B.keys + 6 * c + q, okey(bmin[3 * id + q]));
        atomicMax(B.keys + 6 * c + 3 + q, okey(bmax[3 * id + q]));
      }
    }
  }
}

// SAH sweep of axis k, in the host's order: best cost and cut.
__device__ void sweep_axis(const Bins &B, int k, const double *box, uint32_t nb, double *best,
                           double *cut) {
  const long long *row = B.keys + 6 * size_t(k) * nb;
  const uint32_t *cnt = B.count + size_t(k) * nb;
  double *rc = B.rcost + size_t(k) * nb;
  double amn[3] = {kMax, kMax, kMax}, amx[3] = {-kMax, -kMax, -kMax};
  size_t c = 0;
  for (uint32_t i = nb - 1; i > 0; --i) {  // right-hand costs
    for (int q = 0; q < 3; ++q) {
      const double bmn = ukey(row[6 * i + q]), bmx = ukey(row[6 * i + 3 + q]);
      amn[q] = (amn[q] < bmn) ? amn[q] : bmn;  // std::min(bmn, amn)
      amx[q] = (bmx < amx[q]) ? amx[q] : bmx;  // std::max(bmx, amx)
    }
    c += cnt[i];
    rc[i] = static_cast<double>(c) * surface(amn, amx);
  }
  for (int q = 0; q < 3; ++q) {
    amn[q] = kMax;
    amx[q] = -kMax;
  }
  c = 0;
  uint32_t first_right = 1;
  double bst = kMax;
  for (uint32_t i = 0; i + 1 < nb; ++i) {  // left sweep, full cost
    for (int q = 0; q < 3; ++q) {
      const double bmn = ukey(row[6 * i + q]), bmx = ukey(row[6 * i + 3 + q]);
      amn[q] = (amn[q] < bmn) ? amn[q] : bmn;
      amx[q] = (bmx < amx[q]) ? amx[q] : bmx;
    }
    c += cnt[i];
    const double cost = static_cast<double>(c) * surface(amn, amx) + rc[i + 1];
    if (cost < bst) {
      bst = cost;
      first_right = i + 1;
    }
  }
  best[k] = bst;
  cut[k] = static_cast<double>(first_right) * ((box[3 + k] - box[k]) / static_cast<double>(nb)) +
           box[k];
}

// Block sums of the centres of positions [a, b) below each axis's cut, added into below[3].
__device__ void count_below(const double *ctr, const uint32_t *ids, uint32_t a, uint32_t b,
                            const double *cut, uint32_t *below) {
  const unsigned lane = threadIdx.x & 31u;
  uint32_t mine[3] = {0, 0, 0};
  for (uint32_t i = a + threadIdx.x; i < b; i += blockDim.x) {
    const size_t id = ids[i];
    for (int k = 0; k < 3; ++k) mine[k] += ctr[3 * id + k] < cut[k] ? 1u : 0u;
  }
  for (int k = 0; k < 3; ++k) {
    uint32_t v = mine[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lane == 0 && v) atomicAdd(below + k, v);
  }
}

// The host's axis choice and attempt sequence (blazert/bvh/builder.h:201-226):
// decision = {final axis, axis whose partition applies or 0xFFFFFFFF, left count}.
// Failed attempts are added to counts[3] (the bad-split count).
__device__ void decide(const double *best, const uint32_t *below, uint32_t n, uint32_t *decision,
                       uint32_t *counts) {
  uint32_t axis = 0;
  if (best[0] > best[1]) axis = 1;
  if (best[axis] > best[2]) axis = 2;
  int split_axis = -1;
  uint32_t bad = 0;
  for (int attempt = 0; attempt < 3; ++attempt) {
    const uint32_t m = below[axis];
    if (m == 0 || m == n) {
      ++bad;
      axis = (axis + 1) % 3;
    } else {
      split_axis = static_cast<int>(axis);
      break;
    }
  }
  if (bad) atomicAdd(counts + 3, bad);
  decision[0] = axis;
  decision[1] = static_cast<uint32_t>(split_axis);
  decision[2] = split_axis >= 0 ? below[split_axis] : (n >> 1);
}

// Writes L[l0 + rank] for the failing positions of [a, b) (left to right) and R[r0 + rank] for
// the passing positions of [c, d) (right to left); returns the number of failing positions.
// Block-uniform arguments, a <= b and c <= d.
__device__ uint32_t pair_lists(const double *ctr, const uint32_t *ids, uint32_t *L, uint32_t *R,
                               int axis, double cv, uint32_t a, uint32_t b, uint32_t l0,
                               uint32_t c, uint32_t d, uint32_t r0, uint32_t *warp_sums) {
  uint32_t carry = 0, total = 0;
  for (uint32_t t = a; t < b; t += blockDim.x) {
    const uint32_t i = t + threadIdx.x;
    bool fail = false;
    if (i < b) fail = !(ctr[3 * size_t(ids[i]) + axis] < cv);
    const uint32_t r = block_rank(fail, warp_sums, &total);
    if (fail) L[l0 + carry + r] = i;
    carry += total;
  }
  const uint32_t fails = carry;
  carry = 0;
  for (uint32_t t = 0; t < d - c; t += blockDim.x) {
    const uint32_t j = t + threadIdx.x;  // j-th position from the right end of [c, d)
    bool pass = false;
    uint32_t p = 0;
    if (j < d - c) {
      p = d - 1 - j;
      pass = ctr[3 * size_t(ids[p]) + axis] < cv;
    }
    const uint32_t r = block_rank(pass, warp_sums, &total);
    if (pass) R[r0 + carry + r] = p;
    carry += total;
  }
  return fails;
}

// Swaps ids at L[q] and R[q] for q in [q0, q1): std::partition's exchanges.
__device__ void apply_swaps(uint32_t *ids, const uint32_t *L, const uint32_t *R, uint32_t q0,
                            uint32_t q1) {
  for (uint32_t q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
    const uint32_t a = L[q], b = R[q];
    const uint32_t t = ids[a];
    ids[a] = ids[b];
    ids[b] = t;
  }
}

// Node record and child ranges of a split node (one thread).
__device__ void emit_children(GNode *nd, const Seg &sg, uint32_t axis, uint32_t m,
                              uint32_t *node_count, Seg *next, uint32_t *next_count,
                              Seg *next_wide, uint32_t *next_wide_count) {
  const uint32_t c0 = atomicAdd(node_count, 2u);
  nd->leaf = 0;
  nd->axis = axis;
  nd->child0 = c0;
  nd->child1 = c0 + 1;
  const uint32_t mid = sg.begin + m;
  const Seg kids[2] = {Seg{sg.begin, mid, sg.depth + 1, c0}, Seg{mid, sg.end, sg.depth + 1, c0 + 1}};
  for (const Seg &k : kids) {
    if (k.end - k.begin >= kWidePrims) {
      next_wide[atomicAdd(next_wide_count, 1u)] = k;
    } else {
      next[atomicAdd(next_count, 1u)] = k;
    }
  }
}

struct LevelArgs {
  const double *bmin, *bmax, *ctr;
  uint32_t *ids, *L, *R;
  GNode *nodes;
  uint32_t *counts;  // [0] next ranges, [1] nodes, [2] max depth, [3] bad splits, [4] next wide
  Seg *next, *next_wide;
  uint32_t min_leaf, max_depth, nb;
};

// One CTA per node of the level (ranges below kWidePrims primitives).
__global__ void __launch_bounds__(kThreads) build_level_kernel(LevelArgs A, const Seg *segs) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Bins B = bins_at(smem, A.nb);
  __shared__ double red[2][3][kThreads / 32];
  __shared__ double box[6], cut[3], best[3];
  __shared__ uint32_t below[3], warp_sums[kThreads / 32], decision[3];

  const Seg sg = segs[blockIdx.x];
  const uint32_t n = sg.end - sg.begin;
  box_reduce(A.bmin, A.bmax, A.ids, sg.begin, sg.end, red, box);
  GNode *nd = A.nodes + sg.node;
  if (threadIdx.x == 0) {
    for (int k = 0; k < 3; ++k) {
      nd->mn[k] = box[k];
      nd->mx[k] = box[3 + k];
    }
    nd->begin = sg.begin;
    nd->end = sg.end;
    atomicMax(A.counts + 2, sg.depth);
  }
  if (n <= A.min_leaf || sg.depth >= A.max_depth) {  // leaf (block-uniform)
    if (threadIdx.x == 0) {
      nd->leaf = 1;
      nd->axis = nd->child0 = nd->child1 = 0xFFFFFFFFu;
    }
    return;
  }
  bins_clear(B, A.nb);
  __syncthreads();
  bin_prims(B, A.bmin, A.bmax, A.ctr, A.ids, sg.begin, sg.end, box, A.nb);
  __syncthreads();
  if (threadIdx.x < 3) {
    sweep_axis(B, threadIdx.x, box, A.nb, best, cut);
    below[threadIdx.x] = 0;
  }
  __syncthreads();
  count_below(A.ctr, A.ids, sg.begin, sg.end, cut, below);
  __syncthreads();
  if (threadIdx.x == 0) decide(best, below, n, decision, A.counts);
  __syncthreads();
  const uint32_t axis = decision[0], m = decision[2];
  const int split_axis = static_cast<int>(decision[1]);
  if (split_axis >= 0) {  // std::partition's exchanges
    const uint32_t nbad = pair_lists(A.ctr, A.ids, A.L, A.R, split_axis, cut[split_axis],
                                     sg.begin, sg.begin + m, sg.begin, sg.begin + m, sg.end,
                                     sg.begin, warp_sums);
    __syncthreads();
    apply_swaps(A.ids, A.L, A.R, sg.begin, sg.begin + nbad);
  }
  if (threadIdx.x == 0)
    emit_children(nd, sg, axis, m, A.counts + 1, A.next, A.counts, A.next_wide, A.counts + 4);
}

// One cluster of kCluster CTAs per node of at least kWidePrims primitives: each CTA takes an
// eighth of the range; rank 0 merges the partial boxes, bins and counts from its peers' shared
// memory, sweeps and decides; every CTA then writes its share of the exchange lists (offsets
// from its peers' counts) and performs its share of the exchanges.  Every CTA passes every
// cluster barrier; none exits while a peer may still read its shared memory.
__global__ void __launch_bounds__(kThreads) build_wide_kernel(LevelArgs A, const Seg *segs) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const unsigned rank = cl.block_rank(), C = cl.num_blocks();
  extern __shared__ __align__(16) unsigned char smem[];
  const Bins B = bins_at(smem, A.nb);
  __shared__ double red[2][3][kThreads / 32];
  __shared__ double box[6], gbox[6], cut[3], best[3];
  __shared__ uint32_t below[3], tbelow[3], warp_sums[kThreads / 32], decision[3], part[2];

  const Seg sg = segs[blockIdx.x / C];
  const uint32_t n = sg.end - sg.begin;
  const uint32_t a = sg.begin + uint32_t(uint64_t(n) * rank / C);
  const uint32_t b = sg.begin + uint32_t(uint64_t(n) * (rank + 1) / C);
  // 1. node box: partial per CTA, merged by rank 0
  box_reduce(A.bmin, A.bmax, A.ids, a, b, red, box);
  cl.sync();
  if (rank == 0 && threadIdx.x < 3) {
    const int k = threadIdx.x;
    double lo = box[k], hi = box[3 + k];
    for (unsigned r = 1; r < C; ++r) {
      const double *pb = cl.map_shared_rank(box, r);
      lo = fmin(lo, pb[k]);
      hi = fmax(hi, pb[3 + k]);
    }
    gbox[k] = lo;
    gbox[3 + k] = hi;
  }
  cl.sync();
  if (threadIdx.x < 6) gbox[threadIdx.x] = cl.map_shared_rank(gbox, 0)[threadIdx.x];
  __syncthreads();
  GNode *nd = A.nodes + sg.node;
  if (rank == 0 && threadIdx.x == 0) {
    for (int k = 0; k < 3; ++k) {
      nd->mn[k] = gbox[k];
      nd->mx[k] = gbox[3 + k];
    }
    nd->begin = sg.begin;
    nd->end = sg.end;
    atomicMax(A.counts + 2, sg.depth);
  }
  if (n <= A.min_leaf || sg.depth >= A.max_depth) {  // leaf (uniform over the cluster)
    if (rank == 0 && threadIdx.x == 0) {
      nd->leaf = 1;
      nd->axis = nd->child0 = nd->child1 = 0xFFFFFFFFu;
    }
    cl.sync();
    return;
  }
  // 2. bins: partial per CTA, merged into rank 0's, swept there
  bins_clear(B, A.nb);
  __syncthreads();
  bin_prims(B, A.bmin, A.bmax, A.ctr, A.ids, a, b, gbox, A.nb);
  cl.sync();
  if (rank == 0) {
    for (uint32_t i = threadIdx.x; i < 3 * A.nb; i += blockDim.x) {
      uint32_t c = B.count[i];
      long long k6[6];
      for (int q = 0; q < 6; ++q) k6[q] = B.keys[6 * i + q];
      for (unsigned r = 1; r < C; ++r) {
        const Bins P = bins_at(cl.map_shared_rank(smem, r), A.nb);
        c += P.count[i];
        for (int q = 0; q < 3; ++q) {
          k6[q] = min(k6[q], P.keys[6 * i + q]);
          k6[3 + q] = max(k6[3 + q], P.keys[6 * i + 3 + q]);
        }
      }
      B.count[i] = c;
      for (int q = 0; q < 6; ++q) B.keys[6 * i + q] = k6[q];
    }
    __syncthreads();
    if (threadIdx.x < 3) sweep_axis(B, threadIdx.x, gbox, A.nb, best, cut);
  }
  cl.sync();
  if (threadIdx.x < 3) {
    cut[threadIdx.x] = cl.map_shared_rank(cut, 0)[threadIdx.x];
    below[threadIdx.x] = 0;
  }
  __syncthreads();
  // 3. counts below the cuts: partial per CTA, summed and decided by rank 0
  count_below(A.ctr, A.ids, a, b, cut, below);
  cl.sync();
  if (rank == 0 && threadIdx.x == 0) {
    for (int k = 0; k < 3; ++k) {
      uint32_t t = 0;
      for (unsigned r = 0; r < C; ++r) t += cl.map_shared_rank(below, r)[k];
      tbelow[k] = t;
    }
    decide(best, tbelow, n, decision, A.counts);
  }
  cl.sync();
  if (threadIdx.x < 3) decision[threadIdx.x] = cl.map_shared_rank(decision, 0)[threadIdx.x];
  __syncthreads();
  const uint32_t axis = decision[0], m = decision[2];
  const int split_axis = static_cast<int>(decision[1]);
  // 4. std::partition's exchanges, each CTA for its share of the range
  const uint32_t mid = sg.begin + m;
  const uint32_t fa = a, fb = max(a, min(b, mid));         // its part of [begin, mid)
  const uint32_t pa = min(b, max(a, mid)), pb = b;          // its part of [mid, end)
  const double cv = split_axis >= 0 ? cut[split_axis] : 0.0;
  if (threadIdx.x == 0) part[0] = part[1] = 0;
  __syncthreads();
  if (split_axis >= 0) {
    uint32_t f = 0, p = 0;
    for (uint32_t i = fa + threadIdx.x; i < fb; i += blockDim.x)
      f += !(A.ctr[3 * size_t(A.ids[i]) + split_axis] < cv) ? 1u : 0u;
    for (uint32_t i = pa + threadIdx.x; i < pb; i += blockDim.x)
      p += A.ctr[3 * size_t(A.ids[i]) + split_axis] < cv ? 1u : 0u;
    for (int o = 16; o > 0; o >>= 1) {
      f += __shfl_xor_sync(0xFFFFFFFFu, f, o);
      p += __shfl_xor_sync(0xFFFFFFFFu, p, o);
    }
    if ((threadIdx.x & 31u) == 0) {
      if (f) atomicAdd(part, f);
      if (p) atomicAdd(part + 1, p);
    }
  }
  cl.sync();
  uint32_t l0 = sg.begin, r0 = sg.begin, nbad = 0;
  for (unsigned r = 0; r < C; ++r) {
    const uint32_t *pr = cl.map_shared_rank(part, r);
    if (r < rank) l0 += pr[0];
    if (r > rank) r0 += pr[1];
    nbad += pr[0];
  }
  if (split_axis >= 0)
    pair_lists(A.ctr, A.ids, A.L, A.R, split_axis, cv, fa, fb, l0, pa, pb, r0, warp_sums);
  __threadfence();
  cl.sync();  // the exchange lists are complete, and no peer reads `part` any more
  if (split_axis >= 0)
    apply_swaps(A.ids, A.L, A.R, sg.begin + uint32_t(uint64_t(nbad) * rank / C),
                sg.begin + uint32_t(uint64_t(nbad) * (rank + 1) / C));
  if (rank == 0 && threadIdx.x == 0)
    emit_children(nd, sg, axis, m, A.counts + 1, A.next, A.counts, A.next_wide, A.counts + 4);
}

// DFS pre-order renumbering of the level-order nodes: subtree sizes bottom up, then indices
// top down (node, left subtree, right subtree), then the nodes scattered into that order.
__global__ void subtree_size_kernel(const GNode *g, uint32_t *size, uint32_t lo, uint32_t hi) {
  for (uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi;
       i += gridDim.x * blockDim.x)
    size[i] = g[i].leaf == 1 ? 1u : 1u + size[g[i].child0] + size[g[i].child1];
}
__global__ void dfs_index_kernel(const GNode *g, const uint32_t *size, uint32_t *dfs, uint32_t lo,
                                 uint32_t hi) {
  for (uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi;
       i += gridDim.x * blockDim.x) {
    if (g[i].leaf == 1) continue;
    dfs[g[i].child0] = dfs[i] + 1;
    dfs[g[i].child1] = dfs[i] + 1 + size[g[i].child0];
  }
}
__global__ void scatter_kernel(const GNode *g, const uint32_t *dfs, TreeNode *out, uint32_t count) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += gridDim.x * blockDim.x) {
    const GNode &s = g[i];
    TreeNode t;
    for (int k = 0; k < 3; ++k) {
      t.mn[k] = s.mn[k];
      t.mx[k] = s.mx[k];
    }
    t.leaf = s.leaf;
    t.axis = s.axis;
    const bool leaf = s.leaf == 1;
    t.child[0] = leaf ? 0xFFFFFFFFu : dfs[s.child0];
    t.child[1] = leaf ? 0xFFFFFFFFu : dfs[s.child1];
    t.prim_off = leaf ? s.begin : 0u;
    t.prim_cnt = leaf ? s.end - s.begin : 0u;
    out[dfs[i]] = t;
  }
}

// Device scratch of the builder, one per device, kept from build to build and grown on demand.
// A mesh of 3 x 10^5 triangles builds its levels in about 5 ms, while allocating and releasing
// its scratch (about 420 bytes per primitive) took about 40 ms; a workspace above kKeepBytes is
// released after its build.  The mutex serialises device builds of one process.
constexpr size_t kKeepBytes = size_t(2) << 30;
constexpr int kMaxDevices = 64;
struct Workspace {
  void *ptr = nullptr;
  size_t bytes = 0;
};
std::mutex g_workspace_mutex;
Workspace g_workspace[kMaxDevices];

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

bool finite_boxes(const PrimBoxes &b) {
  for (size_t i = 0; i < 3 * b.n; ++i)
    if (!std::isfinite(b.bmin[i]) || !std::isfinite(b.bmax[i]) || !std::isfinite(b.center[i]))
      return false;
  return true;
}

}  // namespace

bool gpu_build_possible(const PrimBoxes &boxes, const BuildOptions &opt) {
  // min_leaf >= 1 keeps every child range non-empty, which bounds the nodes by 2n - 1 and
  // the ranges of a level by n (the device arrays are sized for that)
  return boxes.n >= 1 && boxes.n < 0x7FFFFFFFu && opt.min_leaf >= 1 && opt.bins >= 2 &&
         opt.bins <= 256 && finite_boxes(boxes);
}

cudaError_t gpu_build_tree(const PrimBoxes &boxes, const BuildOptions &opt, Tree *out) {
  const size_t n = boxes.n;
  const size_t max_nodes = 2 * n;  // 2n - 1 nodes at most with min_leaf >= 1
  const size_t max_wide = n / kWidePrims + 2;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  // bmin, bmax, centre (n x 3 each); ids, L, R, counts[8], size, dfs; narrow ranges x 2 and
  // wide ranges x 2; level-order nodes; DFS-ordered nodes
  const size_t sz_box = align256(72 * n);
  const size_t sz_u32 = align256(sizeof(uint32_t) * (3 * n + 8 + 2 * max_nodes));
  const size_t sz_seg = align256(sizeof(Seg) * 2 * (n + 1 + max_wide));
  const size_t sz_nodes = align256(sizeof(GNode) * max_nodes);
  const size_t need = sz_box + sz_u32 + sz_seg + sz_nodes + sizeof(TreeNode) * max_nodes;
  std::vector<uint32_t> ids(n);
  for (size_t i = 0; i < n; ++i) ids[i] = static_cast<uint32_t>(i);
  Tree &t = *out;
  uint32_t h[8];
  std::unique_lock<std::mutex> lock(g_workspace_mutex);
  Workspace &ws = g_workspace[dev];
  if (ws.bytes < need) {
    if (ws.ptr) cudaFree(ws.ptr);
    ws = Workspace{};
    e = bzr::dev_malloc(&ws.ptr, need);
    if (e != cudaSuccess) {
      ws.ptr = nullptr;
      return e;
    }
    ws.bytes = need;
  }
  char *base = static_cast<char *>(ws.ptr);
  double *d_box = reinterpret_cast<double *>(base);
  uint32_t *d_u32 = reinterpret_cast<uint32_t *>(base + sz_box);
  Seg *d_seg = reinterpret_cast<Seg *>(base + sz_box + sz_u32);
  GNode *d_nodes = reinterpret_cast<GNode *>(base + sz_box + sz_u32 + sz_seg);
  TreeNode *d_tree = reinterpret_cast<TreeNode *>(base + sz_box + sz_u32 + sz_seg + sz_nodes);
  auto ok = [&](cudaError_t r) {
    if (e == cudaSuccess) e = r;
    return e == cudaSuccess;
  };
  uint32_t *d_ids = d_u32, *d_L = d_u32 + n, *d_R = d_u32 + 2 * n, *d_counts = d_u32 + 3 * n;
  uint32_t *d_size = d_counts + 8, *d_dfs = d_size + max_nodes;
  Seg *narrow[2] = {d_seg, d_seg + (n + 1)};
  Seg *wide[2] = {d_seg + 2 * (n + 1), d_seg + 2 * (n + 1) + max_wide};
  ok(cudaMemcpy(d_box, boxes.bmin.data(), 24 * n, cudaMemcpyHostToDevice));
  ok(cudaMemcpy(d_box + 3 * n, boxes.bmax.data(), 24 * n, cudaMemcpyHostToDevice));
  ok(cudaMemcpy(d_box + 6 * n, boxes.center.data(), 24 * n, cudaMemcpyHostToDevice));
  ok(cudaMemcpy(d_ids, ids.data(), 4 * n, cudaMemcpyHostToDevice));
  const Seg root{0u, static_cast<uint32_t>(n), 0u, 0u};
  const bool root_wide = n >= kWidePrims;
  ok(cudaMemcpy(root_wide ? wide[0] : narrow[0], &root, sizeof root, cudaMemcpyHostToDevice));
  const uint32_t nb = opt.bins;
  const size_t smem = bins_bytes(nb);
  if (smem > 48 * 1024) {
    ok(cudaFuncSetAttribute(build_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            int(smem)));
    ok(cudaFuncSetAttribute(build_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            int(smem)));
  }
  LevelArgs A;
  A.bmin = d_box;
  A.bmax = d_box + 3 * n;
  A.ctr = d_box + 6 * n;
  A.ids = d_ids;
  A.L = d_L;
  A.R = d_R;
  A.nodes = d_nodes;
  A.counts = d_counts;
  A.min_leaf = opt.min_leaf;
  A.max_depth = opt.max_depth;
  A.nb = nb;
  // counts: [0] next narrow ranges, [1] nodes, [2] max depth, [3] bad splits, [4] next wide
  const uint32_t h0[8] = {root_wide ? 0u : 1u, 1u, 0u, 0u, root_wide ? 1u : 0u, 0u, 0u, 0u};
  std::memcpy(h, h0, sizeof h);
  std::vector<uint32_t> level_start{0u, 1u};  // node index ranges of the levels
  int cur = 0;
  uint32_t n_narrow = h[0], n_wide = h[4];
  ok(cudaMemcpy(d_counts, h, sizeof h, cudaMemcpyHostToDevice));
  while (e == cudaSuccess && (n_narrow || n_wide)) {
    const uint32_t zero[1] = {0u};
    ok(cudaMemcpy(d_counts, zero, 4, cudaMemcpyHostToDevice));
    ok(cudaMemcpy(d_counts + 4, zero, 4, cudaMemcpyHostToDevice));
    A.next = narrow[cur ^ 1];
    A.next_wide = wide[cur ^ 1];
    if (n_narrow && e == cudaSuccess) {
      build_level_kernel<<<n_narrow, kThreads, smem>>>(A, narrow[cur]);
      ok(cudaGetLastError());
    }
    if (n_wide && e == cudaSuccess) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(n_wide * kCluster);
      cfg.blockDim = dim3(kThreads);
      cfg.dynamicSmemBytes = smem;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = kCluster;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      ok(cudaLaunchKernelEx(&cfg, build_wide_kernel, A, static_cast<const Seg *>(wide[cur])));
    }
    ok(cudaMemcpy(h, d_counts, sizeof h, cudaMemcpyDeviceToHost));
    n_narrow = h[0];
    n_wide = h[4];
    level_start.push_back(h[1]);  // the next level's nodes end here
    cur ^= 1;
  }
  const uint32_t count = h[1];
  if (e == cudaSuccess && count > max_nodes) e = cudaErrorUnknown;
  // level L holds node indices [level_start[L], level_start[L + 1]); the last entry repeats
  const int levels = static_cast<int>(level_start.size()) - 1;
  const int grid = 1024;
  for (int L = levels - 1; L >= 0 && e == cudaSuccess; --L) {
    const uint32_t lo = level_start[L], hi = level_start[L + 1];
    if (hi > lo) subtree_size_kernel<<<grid, 256>>>(d_nodes, d_size, lo, hi);
  }
  ok(cudaGetLastError());
  ok(cudaMemset(d_dfs, 0, 4));  // the root comes first
  for (int L = 0; L < levels && e == cudaSuccess; ++L) {
    const uint32_t lo = level_start[L], hi = level_start[L + 1];
    if (hi > lo) dfs_index_kernel<<<grid, 256>>>(d_nodes, d_size, d_dfs, lo, hi);
  }
  if (e == cudaSuccess) scatter_kernel<<<grid, 256>>>(d_nodes, d_dfs, d_tree, count);
  ok(cudaGetLastError());
  if (e == cudaSuccess) {
    t.nodes.resize(count);
    ok(cudaMemcpy(t.nodes.data(), d_tree, sizeof(TreeNode) * count, cudaMemcpyDeviceToHost));
    ok(cudaMemcpy(ids.data(), d_ids, 4 * n, cudaMemcpyDeviceToHost));
  }
  // nothing of this build may still run on the workspace when the next build takes it
  if (e != cudaSuccess) cudaStreamSynchronize(0);
  if (ws.bytes > kKeepBytes) {
    cudaFree(ws.ptr);
    ws = Workspace{};
  }
  lock.unlock();
  if (e != cudaSuccess) return e;
  // structural check before anything walks the tree: DFS pre-order (left child right after its
  // parent, right child after that), leaf ranges tiling [0, n) left to right
  uint64_t next_prim = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const TreeNode &nd = t.nodes[i];
    if (nd.leaf == 1) {
      if (nd.prim_off != next_prim || nd.prim_cnt == 0) return cudaErrorUnknown;
      next_prim += nd.prim_cnt;
    } else if (nd.leaf != 0 || nd.child[0] != i + 1 || nd.child[1] <= i + 1 ||
               nd.child[1] >= count) {
      return cudaErrorUnknown;
    }
  }
  if (next_prim != n) return cudaErrorUnknown;
  t.leaf_prims = std::move(ids);
  t.max_depth = h[2];
  t.bad_splits = h[3];
  return cudaSuccess;
}

}  // namespace bzr
