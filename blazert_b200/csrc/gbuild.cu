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
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "scene.h"

namespace bzr {
namespace {

constexpr int kThreads = 256;
constexpr double kMax = 1.7976931348623157e308;

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

__global__ void __launch_bounds__(kThreads)
    build_level_kernel(const double *__restrict__ bmin, const double *__restrict__ bmax,
                       const double *__restrict__ ctr, uint32_t *ids, uint32_t *L, uint32_t *R,
                       const Seg *segs, Seg *next, uint32_t *next_count, GNode *nodes,
                       uint32_t *node_count, uint32_t *stats, uint32_t min_leaf,
                       uint32_t max_depth, uint32_t nb) {
  extern __shared__ __align__(16) unsigned char smem[];
  // shared, per axis and bin: 6 ordered box keys, the right-hand cost, the count
  long long *keys = reinterpret_cast<long long *>(smem);              // 3 * nb * 6
  double *rcost = reinterpret_cast<double *>(keys + 18 * size_t(nb));  // 3 * nb
  uint32_t *count = reinterpret_cast<uint32_t *>(rcost + 3 * size_t(nb));  // 3 * nb
  __shared__ double red[2][3][kThreads / 32];
  __shared__ double box[6], cut[3], best[3];
  __shared__ uint32_t below[3], warp_sums[kThreads / 32], decision[3];

  const Seg sg = segs[blockIdx.x];
  const uint32_t n = sg.end - sg.begin;
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;

  // 1. node box
  double mn[3] = {kMax, kMax, kMax}, mx[3] = {-kMax, -kMax, -kMax};
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const size_t id = ids[sg.begin + i];
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
    double a = kMax, b = -kMax;
    for (unsigned w = 0; w < blockDim.x / 32; ++w) {
      a = fmin(a, red[0][k][w]);
      b = fmax(b, red[1][k][w]);
    }
    box[k] = a;
    box[3 + k] = b;
  }
  __syncthreads();
  GNode *nd = nodes + sg.node;
  if (threadIdx.x == 0) {
    for (int k = 0; k < 3; ++k) {
      nd->mn[k] = box[k];
      nd->mx[k] = box[3 + k];
    }
    nd->begin = sg.begin;
    nd->end = sg.end;
    atomicMax(stats, sg.depth);
  }
  // 2. leaf
  if (n <= min_leaf || sg.depth >= max_depth) {
    if (threadIdx.x == 0) {
      nd->leaf = 1;
      nd->axis = nd->child0 = nd->child1 = 0xFFFFFFFFu;
    }
    return;
  }
  // 3. bins
  for (uint32_t i = threadIdx.x; i < 3 * nb; i += blockDim.x) {
    for (int q = 0; q < 3; ++q) {
      keys[6 * i + q] = okey(kMax);
      keys[6 * i + 3 + q] = okey(-kMax);
    }
    count[i] = 0;
  }
  __syncthreads();
  double inv[3];
  for (int k = 0; k < 3; ++k) {
    const double ext = box[3 + k] - box[k];
    inv[k] = ext > 0.0 ? 1.0 / ext : 0.0;
  }
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const size_t id = ids[sg.begin + i];
    for (int k = 0; k < 3; ++k) {
      const double pos = ((ctr[3 * id + k] - box[k]) * inv[k]) * static_cast<double>(nb - 1);
      // the host's min(nb - 1, unsigned(max(0u, unsigned(round(pos))))), with the
      // double -> unsigned conversion going through a 64-bit signed integer
      const unsigned r = static_cast<unsigned>(static_cast<long long>(round(pos)));
      const uint32_t slot = min(nb - 1, max(0u, r));
      const uint32_t b = k * nb + slot;
      atomicAdd(count + b, 1u);
      for (int q = 0; q < 3; ++q) {
        atomicMin(keys + 6 * b + q, okey(bmin[3 * id + q]));
        atomicMax(keys + 6 * b + 3 + q, okey(bmax[3 * id + q]));
      }
    }
  }
  __syncthreads();
  // 4. sweep, one thread per axis, in the host's order
  if (threadIdx.x < 3) {
    const int k = threadIdx.x;
    const long long *row = keys + 6 * size_t(k) * nb;
    const uint32_t *cnt = count + size_t(k) * nb;
    double *rc = rcost + size_t(k) * nb;
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
    below[k] = 0;
  }
  __syncthreads();
  // 5. centres below each axis's cut, and the host's attempt sequence
  uint32_t mine[3] = {0, 0, 0};
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const size_t id = ids[sg.begin + i];
    for (int k = 0; k < 3; ++k) mine[k] += ctr[3 * id + k] < cut[k] ? 1u : 0u;
  }
  for (int k = 0; k < 3; ++k) {
    uint32_t v = mine[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lane == 0 && v) atomicAdd(below + k, v);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t axis = 0;
    if (best[0] > best[1]) axis = 1;
    if (best[axis] > best[2]) axis = 2;
    int split_axis = -1;  // axis whose partition is applied; -1: middle of the range
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
    if (bad) atomicAdd(stats + 1, bad);
    decision[0] = axis;
    decision[1] = static_cast<uint32_t>(split_axis);
    decision[2] = split_axis >= 0 ? below[split_axis] : (n >> 1);
  }
  __syncthreads();
  const uint32_t axis = decision[0];
  const int split_axis = static_cast<int>(decision[1]);
  const uint32_t m = decision[2];
  // 6. std::partition's swaps: the k-th failing element of [0, m) with the k-th passing
  // element of [m, n) counted from the right
  if (split_axis >= 0) {
    const double cv = cut[split_axis];
    uint32_t carry = 0, total = 0;
    for (uint32_t t = 0; t < m; t += blockDim.x) {
      const uint32_t i = t + threadIdx.x;
      bool fail = false;
      if (i < m) fail = !(ctr[3 * size_t(ids[sg.begin + i]) + split_axis] < cv);
      const uint32_t r = block_rank(fail, warp_sums, &total);
      if (fail) L[sg.begin + carry + r] = sg.begin + i;
      carry += total;
    }
    const uint32_t nbad = carry;
    carry = 0;
    for (uint32_t t = 0; t < n - m; t += blockDim.x) {
      const uint32_t j = t + threadIdx.x;  // j-th position from the right end
      bool pass = false;
      uint32_t p = 0;
      if (j < n - m) {
        p = sg.end - 1 - j;
        pass = ctr[3 * size_t(ids[p]) + split_axis] < cv;
      }
      const uint32_t r = block_rank(pass, warp_sums, &total);
      if (pass) R[sg.begin + carry + r] = p;
      carry += total;
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < nbad; q += blockDim.x) {
      const uint32_t a = L[sg.begin + q], b = R[sg.begin + q];
      const uint32_t t = ids[a];
      ids[a] = ids[b];
      ids[b] = t;
    }
  }
  // 7. children
  if (threadIdx.x == 0) {
    const uint32_t c0 = atomicAdd(node_count, 2u);
    nd->leaf = 0;
    nd->axis = axis;
    nd->child0 = c0;
    nd->child1 = c0 + 1;
    const uint32_t s = atomicAdd(next_count, 2u);
    const uint32_t mid = sg.begin + m;
    next[s] = Seg{sg.begin, mid, sg.depth + 1, c0};
    next[s + 1] = Seg{mid, sg.end, sg.depth + 1, c0 + 1};
  }
}

bool finite_boxes(const PrimBoxes &b) {
  for (size_t i = 0; i < 3 * b.n; ++i)
    if (!std::isfinite(b.bmin[i]) || !std::isfinite(b.bmax[i]) || !std::isfinite(b.center[i]))
      return false;
  return true;
}

}  // namespace

bool gpu_build_possible(const PrimBoxes &boxes, const BuildOptions &opt) {
  return boxes.n >= 1 && boxes.n < 0x7FFFFFFFu && opt.bins >= 2 && opt.bins <= 256 &&
         finite_boxes(boxes);
}

cudaError_t gpu_build_tree(const PrimBoxes &boxes, const BuildOptions &opt, Tree *out) {
  const size_t n = boxes.n;
  const size_t max_nodes = 2 * n + 1;
  double *d_bmin = nullptr, *d_bmax = nullptr, *d_ctr = nullptr;
  uint32_t *d_ids = nullptr, *d_L = nullptr, *d_R = nullptr, *d_counts = nullptr;
  Seg *d_seg[2] = {nullptr, nullptr};
  GNode *d_nodes = nullptr;
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t r) {
    if (e == cudaSuccess) e = r;
    return e == cudaSuccess;
  };
  ok(cudaMalloc(&d_bmin, 24 * n));
  ok(cudaMalloc(&d_bmax, 24 * n));
  ok(cudaMalloc(&d_ctr, 24 * n));
  ok(cudaMalloc(&d_ids, 4 * n));
  ok(cudaMalloc(&d_L, 4 * n));
  ok(cudaMalloc(&d_R, 4 * n));
  ok(cudaMalloc(&d_counts, 16));  // next_count, node_count, max depth, bad splits
  ok(cudaMalloc(&d_seg[0], sizeof(Seg) * (n + 1)));
  ok(cudaMalloc(&d_seg[1], sizeof(Seg) * (n + 1)));
  ok(cudaMalloc(&d_nodes, sizeof(GNode) * max_nodes));
  std::vector<uint32_t> ids(n);
  for (size_t i = 0; i < n; ++i) ids[i] = static_cast<uint32_t>(i);
  ok(cudaMemcpy(d_bmin, boxes.bmin.data(), 24 * n, cudaMemcpyHostToDevice));
  ok(cudaMemcpy(d_bmax, boxes.bmax.data(), 24 * n, cudaMemcpyHostToDevice));
  ok(cudaMemcpy(d_ctr, boxes.center.data(), 24 * n, cudaMemcpyHostToDevice));
  ok(cudaMemcpy(d_ids, ids.data(), 4 * n, cudaMemcpyHostToDevice));
  const uint32_t init[4] = {0u, 1u, 0u, 0u};
  ok(cudaMemcpy(d_counts, init, sizeof init, cudaMemcpyHostToDevice));
  const Seg root{0u, static_cast<uint32_t>(n), 0u, 0u};
  ok(cudaMemcpy(d_seg[0], &root, sizeof root, cudaMemcpyHostToDevice));
  const uint32_t nb = opt.bins;
  const size_t smem = (8 * 18 + 8 * 3 + 4 * 3) * size_t(nb);
  if (e == cudaSuccess && smem > 48 * 1024)
    ok(cudaFuncSetAttribute(build_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            int(smem)));
  uint32_t nseg = 1;
  int cur = 0;
  while (e == cudaSuccess && nseg > 0) {
    ok(cudaMemset(d_counts, 0, sizeof(uint32_t)));  // next_count
    build_level_kernel<<<nseg, kThreads, smem>>>(d_bmin, d_bmax, d_ctr, d_ids, d_L, d_R,
                                                 d_seg[cur], d_seg[cur ^ 1], d_counts,
                                                 d_nodes, d_counts + 1, d_counts + 2,
                                                 opt.min_leaf, opt.max_depth, nb);
    ok(cudaGetLastError());
    ok(cudaMemcpy(&nseg, d_counts, sizeof nseg, cudaMemcpyDeviceToHost));
    cur ^= 1;
  }
  uint32_t counts[4] = {0, 0, 0, 0};
  ok(cudaMemcpy(counts, d_counts, sizeof counts, cudaMemcpyDeviceToHost));
  std::vector<GNode> g(counts[1]);
  if (e == cudaSuccess && counts[1] <= max_nodes) {
    ok(cudaMemcpy(g.data(), d_nodes, sizeof(GNode) * g.size(), cudaMemcpyDeviceToHost));
    ok(cudaMemcpy(ids.data(), d_ids, 4 * n, cudaMemcpyDeviceToHost));
  }
  cudaFree(d_bmin);
  cudaFree(d_bmax);
  cudaFree(d_ctr);
  cudaFree(d_ids);
  cudaFree(d_L);
  cudaFree(d_R);
  cudaFree(d_counts);
  cudaFree(d_seg[0]);
  cudaFree(d_seg[1]);
  cudaFree(d_nodes);
  if (e != cudaSuccess) return e;
  if (counts[1] > max_nodes) return cudaErrorUnknown;
  // DFS pre-order renumbering (node, left subtree, right subtree), as the host recursion
  // creates them; leaves own their range of the final id array
  Tree &t = *out;
  t.nodes.clear();
  t.nodes.reserve(g.size());
  t.leaf_prims = std::move(ids);
  t.max_depth = counts[2];
  t.bad_splits = counts[3];
  std::vector<std::pair<uint32_t, uint32_t>> stack;  // (level-order node, DFS parent slot)
  stack.push_back({0u, 0xFFFFFFFFu});
  std::vector<uint32_t> parent_slot;
  while (!stack.empty()) {
    const auto [gi, pslot] = stack.back();
    stack.pop_back();
    const GNode &src = g[gi];
    const auto self = static_cast<uint32_t>(t.nodes.size());
    if (pslot != 0xFFFFFFFFu) t.nodes[pslot >> 1].child[pslot & 1u] = self;
    TreeNode nd{};
    std::memcpy(nd.mn, src.mn, sizeof nd.mn);
    std::memcpy(nd.mx, src.mx, sizeof nd.mx);
    nd.leaf = src.leaf;
    nd.axis = src.axis;
    nd.child[0] = nd.child[1] = 0xFFFFFFFFu;
    if (src.leaf == 1) {
      nd.prim_off = src.begin;
      nd.prim_cnt = src.end - src.begin;
    } else {
      nd.prim_off = nd.prim_cnt = 0;
    }
    t.nodes.push_back(nd);
    if (src.leaf != 1) {  // right pushed first so that the left subtree is numbered first
      stack.push_back({src.child1, (self << 1) | 1u});
      stack.push_back({src.child0, self << 1});
    }
  }
  return cudaSuccess;
}

}  // namespace bzr
