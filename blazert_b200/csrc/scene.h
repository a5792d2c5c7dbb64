// Host side of a scene: the primitive collections with their precomputed boxes and centres,
// the binned-SAH builder that reproduces the reference's tree node for node, and the
// flattening into the device layout of layout.h.
#pragma once
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "layout.h"

namespace bzr {

// Allocator whose value-less construct leaves an element default-initialised: resize() on a
// vector of numbers then allocates without writing, for arrays that are written in full
// right after (by several threads, which then also take the page faults in parallel).
template <class T>
struct UninitAllocator : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = UninitAllocator<U>;
  };
  UninitAllocator() = default;
#ifdef BZR_POISON_RAW  // test builds: new storage filled with 0xA5, so an unwritten element shows
  T *allocate(size_t n) {
    T *p = std::allocator<T>::allocate(n);
    std::memset(static_cast<void *>(p), 0xA5, n * sizeof(T));
    return p;
  }
#endif
  template <class U>
  UninitAllocator(const UninitAllocator<U> &) noexcept {}
  template <class U>
  void construct(U *p) {
    ::new (static_cast<void *>(p)) U;
  }
  template <class U, class... A>
  void construct(U *p, A &&...a) {
    ::new (static_cast<void *>(p)) U(std::forward<A>(a)...);
  }
};
template <class T>
using RawVector = std::vector<T, UninitAllocator<T>>;

// Worker count for n items at min_per_thread items or more per worker, at most cap.
inline size_t range_workers(size_t n, size_t min_per_thread, size_t cap) {
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  return std::max<size_t>(1, std::min({hw, cap, n / min_per_thread}));
}

// Runs body(begin, end, w) over [0, n) split into `workers` contiguous ranges.  Range 0 runs
// on the calling thread, and so does any range whose thread cannot be started.
template <class F>
void run_ranges(size_t n, size_t workers, const F &body) {
  auto lo = [&](size_t w) { return n * w / workers; };
  std::vector<std::thread> th;
  th.reserve(workers);  // no reallocation below: a failed start leaves every thread joinable
  try {
    for (size_t w = 1; w < workers; ++w) th.emplace_back([&, w] { body(lo(w), lo(w + 1), w); });
  } catch (...) {  // no thread (or no memory for its state): the rest runs here
  }
  body(lo(0), lo(1), 0);
  for (size_t w = th.size() + 1; w < workers; ++w) body(lo(w), lo(w + 1), w);
  for (std::thread &x : th) x.join();
}

struct BuildOptions {
  uint32_t min_leaf = 4;  // blazert/bvh/options.h:20-21 defaults
  uint32_t max_depth = 28;
  uint32_t bins = 64;
};

// Per-primitive boxes and centres of one collection, n x 3 each.
struct PrimBoxes {
  size_t n = 0;
  RawVector<double> bmin, bmax, center;  // every element written by the collection's adder
};

// The reference tree (blazert/bvh/node.h:15-41) in its DFS pre-order.
struct TreeNode {
  double mn[3], mx[3];
  uint32_t leaf, axis, child[2];
  uint32_t prim_off, prim_cnt;  // into Tree::leaf_prims for leaves
};

struct Tree {
  RawVector<TreeNode> nodes;  // every node written by the builder or reader that fills it
  std::vector<uint32_t> leaf_prims;  // primitive ids, leaves in node order
  uint32_t max_depth = 0;
  uint32_t bad_splits = 0;
  double build_seconds = 0.0;
};

Tree build_tree(const PrimBoxes &boxes, const BuildOptions &opt);

// The reference's BVHBuildStatistics (blazert/bvh/statistics.h:11-38, filled by
// bvh/builder.h:84-226) of a built tree: deepest node, leaf and branch counts, fewest and most
// primitives in a leaf (UINT32_MAX / 0 without leaves), failed partition attempts.
struct BuildStatistics {
  uint32_t max_tree_depth = 0, leaf_nodes = 0, max_num_prims_per_leaf = 0;
  uint32_t min_num_prims_per_leaf = 0xFFFFFFFFu, branch_nodes = 0, bad_splits = 0;
};
BuildStatistics tree_statistics(const Tree &t);

// The same tree built on the current CUDA device (gbuild.cu): level by level, one CTA per
// node.  Possible for finite boxes and centres, at least one primitive, min_leaf >= 1 and at
// most 256 bins;
// returns a CUDA error otherwise or on failure (the caller then builds on the host).
bool gpu_build_possible(const PrimBoxes &boxes, const BuildOptions &opt);
cudaError_t gpu_build_tree(const PrimBoxes &boxes, const BuildOptions &opt, Tree *out);

// Host copy of one collection (the caller's arrays are copied at add time).
struct Collection {
  bool present = false;
  uint32_t geom_id = 0xFFFFFFFFu;
  size_t n = 0;
  std::vector<double> a, b, c, d, e;  // kind-specific raw arrays (see scene.cpp)
  PrimBoxes boxes;
  Tree tree;
};

struct HostScene {
  Collection kind[kNumKinds];
  std::vector<double> vertices;   // mesh: n_vertices x 3
  std::vector<uint32_t> faces;    // mesh: n_faces x 3
  std::vector<double> vert_n;     // mesh: accumulated vertex normals
  uint32_t geometries = 0;
  bool committed = false;
  BuildOptions opt;
};

// Collection constructors: copy and precompute (blazert/primitives/*.h collection ctors).
void add_mesh(HostScene &s, const double *v, size_t nv, const uint32_t *f, size_t nf);
void add_spheres(HostScene &s, const double *c, const double *r, size_t n);
void add_planes(HostScene &s, const double *c, const double *dx, const double *dy,
                const double *rot, size_t n);
void add_cylinders(HostScene &s, const double *c, const double *a, const double *b,
                   const double *h, const double *rot, size_t n);

// Device image of one kind, ready to upload.  flatten writes every element of the RawVector
// arrays.
struct KindImage {
  RawVector<double> nodes64;
  std::vector<double> payload;
  RawVector<uint32_t> prim_ids;
  std::vector<uint32_t> pos_of;  // leaf-ordered position of each primitive id
  RawVector<uint32_t> tri;       // triangles: {i0, i1, i2, id word} per leaf-ordered triangle
  RawVector<double> verts;       // triangles: {x, y, z, 0} per vertex, in order of first use
  RawVector<double> vnorm;       // triangles: {nx, ny, nz, 0}, the vertex normal of each vertex
                                 // of verts (same numbering)
  uint32_t n_internal = 0;
  uint32_t root_ref = 0;
  double root_box[6] = {0, 0, 0, 0, 0, 0};
  // mixed-precision image (layout.h, kWideBytes): wide nodes and leaf records
  std::vector<unsigned char> wide;
  RawVector<double> leaves;     // every element written by build_wide
  uint32_t n_wide = 0, n_leaf16 = 0;
  uint32_t wide_root_ref = 0;
  uint32_t wide_stack = 0;      // most stack entries the wide traversal can hold
  float wide_coord_max = 0.0f;  // largest |quantised bound| of the wide nodes, rounded up
  float coord_max = 0.0f;       // largest |coordinate| of the root box, rounded up
  bool mixed_ok = true;         // the wide image was built
};

// Builds the mixed-precision image of a flattened kind (called by flatten).
void build_wide(const Tree &t, int kind, const std::vector<uint32_t> &leaf_pos, KindImage *img);

// Device image of one kind's tree and primitives.  Long loops run on up to max_workers threads;
// the image does not depend on how many.
KindImage flatten(const HostScene &s, int kind, size_t max_workers = 16);

// Persistent scene format (scene_io.cpp): a committed scene's inputs, build options and trees
// as bytes, and back.  decode_scene fills a fresh HostScene (primitives added, trees checked
// and attached, not committed) or returns why the bytes were refused.
RawVector<uint8_t> encode_scene(const HostScene &s);
std::string decode_scene(const uint8_t *data, size_t size, HostScene *out);

// Wavefront OBJ mesh as the reference's examples build it (obj.cpp): vertices n x 3, faces
// m x 3; returns "" or the reason the file was refused.
std::string load_obj(const std::string &path, std::vector<double> *vertices,
                     std::vector<uint32_t> *faces);

}  // namespace bzr
