// Host side of a scene: precompute, binned-SAH build, flattening (see scene.h).
//
// Compiled with -ffp-contract=off.  The precomputed boxes, centres and normals, and every
// decision of the builder, must be bit-identical to the reference's, because the GPU path is
// required to return the reference's prim_id for every ray.  Vector arithmetic follows one
// fixed order throughout: dot = (x0*y0 + x1*y1) + x2*y2, |v| = sqrt(dot(v, v)),
// normalize(v) = v * (1/|v|), (R v)_i = (R_i0 v0 + R_i1 v1) + R_i2 v2.
#include "scene.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>
#include <memory>
#include <numeric>
#include <system_error>
#include <thread>

namespace bzr {
namespace {

constexpr double kMax = std::numeric_limits<double>::max();

struct V3 {
  double x, y, z;
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 load3(const double *p) { return {p[0], p[1], p[2]}; }
inline void store3(double *p, V3 v) {
  p[0] = v.x;
  p[1] = v.y;
  p[2] = v.z;
}
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 normalize(V3 a) {
  const double len = std::sqrt(dot(a, a));
  return scale(a, len != 0.0 ? 1.0 / len : 0.0);
}
inline V3 rotate(const double *R, V3 v) {
  return {(R[0] * v.x + R[1] * v.y) + R[2] * v.z, (R[3] * v.x + R[4] * v.y) + R[5] * v.z,
          (R[6] * v.x + R[7] * v.y) + R[8] * v.z};
}

// Grow the box (mn, mx) by (bmn, bmx) with std::min / std::max argument order of the
// reference's box union (blazert/datatypes.h:87-93).
inline void grow(double *mn, double *mx, const double *bmn, const double *bmx) {
  for (int k = 0; k < 3; ++k) {
    mn[k] = std::min(bmn[k], mn[k]);
    mx[k] = std::max(bmx[k], mx[k]);
  }
}

void alloc_boxes(PrimBoxes &b, size_t n) {
  b.n = n;
  b.bmin.resize(3 * n);
  b.bmax.resize(3 * n);
  b.center.resize(3 * n);
}

// Box of six points, reduced with std::min / std::max over an initializer list as the
// plane and cylinder collections do (first extreme value wins).
void six_point_box(const V3 (&p)[6], double *mn, double *mx) {
  for (int k = 0; k < 3; ++k) {
    mn[k] = std::min({p[0][k], p[1][k], p[2][k], p[3][k], p[4][k], p[5][k]});
    mx[k] = std::max({p[0][k], p[1][k], p[2][k], p[3][k], p[4][k], p[5][k]});
  }
}

// ------------------------------------------------------------------------------ builder
struct Bin {
  double mn[3], mx[3];
  uint32_t count;
  double cost;
  void clear() {
    mn[0] = mn[1] = mn[2] = kMax;
    mx[0] = mx[1] = mx[2] = -kMax;
    count = 0;
    cost = 0.0;
  }
};

// Surface area of a box as the reference computes it (blazert/bvh/binbuffer.h:16-19).
inline double surface(const double *mn, const double *mx) {
  const double e0 = std::abs(mx[0] - mn[0]), e1 = std::abs(mx[1] - mn[1]),
               e2 = std::abs(mx[2] - mn[2]);
  return 2.0 * ((e0 * e1 + e1 * e2) + e2 * e0);
}

// Subtrees of at least this many primitives may be built on another thread.
constexpr uint32_t kParallelPrims = 1u << 15;

class SahBuilder {
 public:
  SahBuilder(const PrimBoxes &p, const BuildOptions &o, Tree &t, std::atomic<int> *threads)
      : p_(p), o_(o), t_(t), bins_(3 * size_t(o.bins)), threads_(threads) {}

  // Returns the index of the node created for [begin, end) (blazert/bvh/builder.h:84-115).
  uint32_t node(uint32_t *begin, uint32_t *end, uint32_t depth) {
    const auto self = static_cast<uint32_t>(t_.nodes.size());
    t_.max_depth = std::max(t_.max_depth, depth);
    t_.nodes.emplace_back();
    TreeNode nd{};
    nd.leaf = nd.axis = nd.child[0] = nd.child[1] = 0xFFFFFFFFu;
    for (int k = 0; k < 3; ++k) {
      nd.mn[k] = kMax;
      nd.mx[k] = -kMax;
    }
    for (const uint32_t *it = begin; it != end; ++it)
      grow(nd.mn, nd.mx, &p_.bmin[3 * *it], &p_.bmax[3 * *it]);
    const auto n = static_cast<uint32_t>(end - begin);
    if (n <= o_.min_leaf || depth >= o_.max_depth) {
      nd.leaf = 1;
      nd.prim_off = static_cast<uint32_t>(t_.leaf_prims.size());
      nd.prim_cnt = n;
      t_.leaf_prims.insert(t_.leaf_prims.end(), begin, end);
      t_.nodes[self] = nd;
      return self;
    }
    uint32_t *mid = nullptr;
    nd.leaf = 0;
    nd.axis = split(begin, end, nd.mn, nd.mx, mid);
    nd.prim_off = nd.prim_cnt = 0;
    t_.nodes[self] = nd;
    // The two halves of the id range are disjoint, so a large right subtree can be built on
    // another thread into its own fragment while this thread builds the left one; splicing
    // the fragment after the left subtree gives the same DFS pre-order node numbering and leaf
    // order as the sequential recursion.
    std::future<Tree> right;
    if (threads_ && static_cast<uint32_t>(end - mid) >= kParallelPrims) {
      if (threads_->fetch_sub(1) > 0) {
        try {
          right = std::async(std::launch::async, [this, mid, end, depth] {
            Tree frag;
            SahBuilder b(p_, o_, frag, threads_);
            b.node(mid, end, depth + 1);
            threads_->fetch_add(1);
            return frag;
          });
        } catch (const std::system_error &) {  // no thread available: build it here
          threads_->fetch_add(1);
        }
      } else {
        threads_->fetch_add(1);  // no thread left: undo the claim
      }
    }
    const uint32_t c0 = node(begin, mid, depth + 1);
    t_.nodes[self].child[0] = c0;
    if (right.valid()) {
      t_.nodes[self].child[1] = splice(right.get());
    } else {
      const uint32_t c1 = node(mid, end, depth + 1);
      t_.nodes[self].child[1] = c1;
    }
    return self;
  }

 private:
  // Binned SAH split (blazert/bvh/binbuffer.h:66-167) followed by the partition with its
  // middle-split fallback that tries the next axis (blazert/bvh/builder.h:201-226).
  uint32_t split(uint32_t *begin, uint32_t *end, const double *mn, const double *mx,
                 uint32_t *&mid) {
    const uint32_t nb = o_.bins;
    for (auto &b : bins_) b.clear();
    double inv[3];
    for (int k = 0; k < 3; ++k) {
      const double ext = mx[k] - mn[k];
      inv[k] = ext > 0.0 ? 1.0 / ext : 0.0;
    }
    for (const uint32_t *it = begin; it != end; ++it) {
      const double *c = &p_.center[3 * *it];
      for (int k = 0; k < 3; ++k) {
        const double pos = ((c[k] - mn[k]) * inv[k]) * static_cast<double>(nb - 1);
        const uint32_t slot =
            std::min(nb - 1, unsigned(std::max(0u, unsigned(std::round(pos)))));
        Bin &b = bins_[k * nb + slot];
        ++b.count;
        grow(b.mn, b.mx, &p_.bmin[3 * *it], &p_.bmax[3 * *it]);
      }
    }
    double cut[3];
    double best[3] = {kMax, kMax, kMax};
    for (int k = 0; k < 3; ++k) {
      Bin *row = &bins_[k * nb];
      double amn[3] = {kMax, kMax, kMax}, amx[3] = {-kMax, -kMax, -kMax};
      size_t count = 0;
      for (uint32_t i = nb - 1; i > 0; --i) {  // right-hand costs
        grow(amn, amx, row[i].mn, row[i].mx);
        count += row[i].count;
        row[i].cost = static_cast<double>(count) * surface(amn, amx);
      }
      for (int q = 0; q < 3; ++q) {
        amn[q] = kMax;
        amx[q] = -kMax;
      }
      count = 0;
      uint32_t first_right = 1;
      for (uint32_t i = 0; i + 1 < nb; ++i) {  // left sweep, full cost
        grow(amn, amx, row[i].mn, row[i].mx);
        count += row[i].count;
        const double cost = static_cast<double>(count) * surface(amn, amx) + row[i + 1].cost;
        if (cost < best[k]) {
          best[k] = cost;
          first_right = i + 1;
        }
      }
      cut[k] = static_cast<double>(first_right) * ((mx[k] - mn[k]) / static_cast<double>(nb)) +
               mn[k];
    }
    uint32_t axis = 0;
    if (best[0] > best[1]) axis = 1;
    if (best[axis] > best[2]) axis = 2;
    for (int attempt = 0; attempt < 3; ++attempt) {
      const double pos = cut[axis];
      const double *ctr = p_.center.data();
      const uint32_t ax = axis;
      mid = std::partition(begin, end,
                           [ctr, ax, pos](uint32_t id) { return ctr[3 * id + ax] < pos; });
      if (mid == begin || mid == end) {
        ++t_.bad_splits;
        mid = begin + ((end - begin) >> 1);
        axis = (axis + 1) % 3;
      } else {
        break;
      }
    }
    return axis;
  }

  // Appends a subtree built as its own fragment (root at index 0); returns its root index.
  uint32_t splice(Tree &&f) {
    const auto base = static_cast<uint32_t>(t_.nodes.size());
    const auto pbase = static_cast<uint32_t>(t_.leaf_prims.size());
    for (TreeNode nd : f.nodes) {
      if (nd.leaf == 1) {
        nd.prim_off += pbase;
      } else {
        nd.child[0] += base;
        nd.child[1] += base;
      }
      t_.nodes.push_back(nd);
    }
    t_.leaf_prims.insert(t_.leaf_prims.end(), f.leaf_prims.begin(), f.leaf_prims.end());
    t_.max_depth = std::max(t_.max_depth, f.max_depth);
    t_.bad_splits += f.bad_splits;
    return base;
  }

  const PrimBoxes &p_;
  const BuildOptions &o_;
  Tree &t_;
  std::vector<Bin> bins_;
  std::atomic<int> *threads_;  // threads that may still be started
};

// Outward rounding of a double bound to float.
inline float round_down(double d) {
  float f = static_cast<float>(d);
  if (static_cast<double>(f) > d) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
  return f;
}
inline float round_up(double d) {
  float f = static_cast<float>(d);
  if (static_cast<double>(f) < d) f = std::nextafter(f, std::numeric_limits<float>::infinity());
  return f;
}

// Long host loops (adding a mesh, flattening) split into contiguous ranges, one per worker
// thread, each range at least this long.
constexpr size_t kNodesPerRange = size_t(1) << 15;
constexpr size_t kPrimsPerRange = size_t(1) << 16;
constexpr size_t kFacesPerRange = size_t(1) << 14;
constexpr size_t kMaxRangeWorkers = 16;

// Mesh part of the image: the vertices numbered in order of first use by the leaf-ordered
// triangles (use u = 3 at + j for corner j of the triangle at position at), stored once each
// with their vertex normals in the same numbering, and per triangle {i0, i1, i2, id word}.  With several workers this takes four passes over
// ranges of triangles: the first use of every vertex (an atomic minimum), the number of first
// uses in each range, the vertex numbers from the prefix sums of those counts, and the
// triangles' indices.  Both ways give the same numbering.
void number_vertices(const HostScene &s, KindImage *img, size_t workers) {
  const size_t np = img->prim_ids.size(), nv = s.vertices.size() / 3;
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  img->tri.resize(4 * np);
  if (workers <= 1 || 3 * uint64_t(np) >= kNone) {
    std::vector<uint32_t> remap(nv, kNone);
    img->verts.reserve(kVertexDoubles * std::min(nv, 3 * np));
    img->vnorm.reserve(kVertexDoubles * std::min(nv, 3 * np));
    for (size_t at = 0; at < np; ++at) {
      const uint32_t *F = &s.faces[3 * size_t(img->prim_ids[at] & kIdMask)];
      for (int j = 0; j < 3; ++j) {
        uint32_t &r = remap[F[j]];
        if (r == kNone) {
          r = static_cast<uint32_t>(img->verts.size() / kVertexDoubles);
          const double *v = &s.vertices[3 * size_t(F[j])];
          img->verts.insert(img->verts.end(), {v[0], v[1], v[2], 0.0});
          const double *vn = &s.vert_n[3 * size_t(F[j])];
          img->vnorm.insert(img->vnorm.end(), {vn[0], vn[1], vn[2], 0.0});
        }
        img->tri[4 * at + j] = r;
      }
      img->tri[4 * at + 3] = img->prim_ids[at];
    }
    return;
  }
  auto corners = [&](size_t at) { return &s.faces[3 * size_t(img->prim_ids[at] & kIdMask)]; };
  std::unique_ptr<std::atomic<uint32_t>[]> first(new std::atomic<uint32_t>[nv]);
  run_ranges(nv, workers, [&](size_t v0, size_t v1, size_t) {
    for (size_t v = v0; v < v1; ++v) first[v].store(kNone, std::memory_order_relaxed);
  });
  run_ranges(np, workers, [&](size_t a0, size_t a1, size_t) {
    for (size_t at = a0; at < a1; ++at) {
      const uint32_t *F = corners(at);
      for (int j = 0; j < 3; ++j) {
        const auto u = static_cast<uint32_t>(3 * at + j);
        std::atomic<uint32_t> &slot = first[F[j]];
        uint32_t cur = slot.load(std::memory_order_relaxed);
        while (u < cur && !slot.compare_exchange_weak(cur, u, std::memory_order_relaxed)) {
        }
      }
    }
  });
  std::vector<size_t> base(workers + 1, 0);
  run_ranges(np, workers, [&](size_t a0, size_t a1, size_t w) {
    size_t n = 0;
    for (size_t at = a0; at < a1; ++at) {
      const uint32_t *F = corners(at);
      for (int j = 0; j < 3; ++j)
        n += first[F[j]].load(std::memory_order_relaxed) == 3 * at + j;
    }
    base[w + 1] = n;
  });
  for (size_t w = 0; w < workers; ++w) base[w + 1] += base[w];
  img->verts.resize(kVertexDoubles * base[workers]);
  img->vnorm.resize(kVertexDoubles * base[workers]);
  RawVector<uint32_t> number(nv);  // read only for the vertices numbered below
  run_ranges(np, workers, [&](size_t a0, size_t a1, size_t w) {
    auto r = static_cast<uint32_t>(base[w]);
    for (size_t at = a0; at < a1; ++at) {
      const uint32_t *F = corners(at);
      for (int j = 0; j < 3; ++j) {
        if (first[F[j]].load(std::memory_order_relaxed) != 3 * at + j) continue;
        number[F[j]] = r;
        const double *v = &s.vertices[3 * size_t(F[j])];
        double *o = &img->verts[kVertexDoubles * size_t(r)];
        o[0] = v[0];
        o[1] = v[1];
        o[2] = v[2];
        o[3] = 0.0;
        const double *vn = &s.vert_n[3 * size_t(F[j])];
        double *on = &img->vnorm[kVertexDoubles * size_t(r)];
        on[0] = vn[0];
        on[1] = vn[1];
        on[2] = vn[2];
        on[3] = 0.0;
        ++r;
      }
    }
  });
  run_ranges(np, workers, [&](size_t a0, size_t a1, size_t) {
    for (size_t at = a0; at < a1; ++at) {
      const uint32_t *F = corners(at);
      for (int j = 0; j < 3; ++j) img->tri[4 * at + j] = number[F[j]];
      img->tri[4 * at + 3] = img->prim_ids[at];
    }
  });
}

}  // namespace

// blazert/bvh/builder.h:46-65
Tree build_tree(const PrimBoxes &boxes, const BuildOptions &opt) {
  Tree t;
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<uint32_t> ids(boxes.n);
  std::iota(ids.begin(), ids.end(), 0u);
  t.nodes.reserve(2 * boxes.n + 1);
  t.leaf_prims.reserve(boxes.n);
  const unsigned hw = std::thread::hardware_concurrency();
  std::atomic<int> threads{hw > 1 ? static_cast<int>(hw) - 1 : 0};
  SahBuilder b(boxes, opt, t, &threads);
  b.node(ids.data(), ids.data() + ids.size(), 0);
  t.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return t;
}

// blazert/primitives/trimesh.h:78-130: centre (v0+v1+v2)/3, box of the corners, unit face
// normal of cross(v1-v0, v2-v0) accumulated /3 into each corner's vertex normal.  The
// per-face values are computed over ranges of faces on several threads; the accumulation
// stays one pass in face order, so each vertex normal is the same sum in the same order.
void add_mesh(HostScene &s, const double *v, size_t nv, const uint32_t *f, size_t nf) {
  Collection &c = s.kind[kMesh];
  s.vertices.assign(v, v + 3 * nv);
  s.faces.assign(f, f + 3 * nf);
  s.vert_n.assign(3 * nv, 0.0);
  c.n = nf;
  alloc_boxes(c.boxes, nf);
  auto face = [&](size_t i) {
    const uint32_t *F = &s.faces[3 * i];
    const V3 a = load3(&s.vertices[3 * size_t(F[0])]), b = load3(&s.vertices[3 * size_t(F[1])]),
             cc = load3(&s.vertices[3 * size_t(F[2])]);
    store3(&c.boxes.center[3 * i], ((a + b) + cc) / 3.0);
    double mn[3] = {a.x, a.y, a.z}, mx[3] = {a.x, a.y, a.z};
    const double pb[3] = {b.x, b.y, b.z}, pc[3] = {cc.x, cc.y, cc.z};
    grow(mn, mx, pb, pb);
    grow(mn, mx, pc, pc);
    std::memcpy(&c.boxes.bmin[3 * i], mn, sizeof mn);
    std::memcpy(&c.boxes.bmax[3 * i], mx, sizeof mx);
    return normalize(cross(b - a, cc - a)) / 3.0;
  };
  auto accumulate = [&](size_t i, V3 share) {
    for (int j = 0; j < 3; ++j) {
      double *vn = &s.vert_n[3 * size_t(s.faces[3 * i + j])];
      store3(vn, load3(vn) + share);
    }
  };
  const size_t workers = range_workers(nf, kFacesPerRange, kMaxRangeWorkers);
  if (workers == 1) {
    for (size_t i = 0; i < nf; ++i) accumulate(i, face(i));
    return;
  }
  RawVector<double> share(3 * nf);
  run_ranges(nf, workers, [&](size_t i0, size_t i1, size_t) {
    for (size_t i = i0; i < i1; ++i) store3(&share[3 * i], face(i));
  });
  for (size_t i = 0; i < nf; ++i) accumulate(i, load3(&share[3 * i]));
}

// blazert/primitives/sphere.h:93-100: box = centre -+ radius.
void add_spheres(HostScene &s, const double *ctr, const double *r, size_t n) {
  Collection &c = s.kind[kSpheres];
  c.n = n;
  c.a.assign(ctr, ctr + 3 * n);
  c.b.assign(r, r + n);
  alloc_boxes(c.boxes, n);
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      c.boxes.bmin[3 * i + k] = c.a[3 * i + k] - c.b[i];
      c.boxes.bmax[3 * i + k] = c.a[3 * i + k] + c.b[i];
      c.boxes.center[3 * i + k] = c.a[3 * i + k];
    }
}

// blazert/primitives/plane.h:113-150: box of the four rotated corners and the two points
// +-DBL_MIN along the rotated normal.
void add_planes(HostScene &s, const double *ctr, const double *dx, const double *dy,
                const double *rot, size_t n) {
  Collection &c = s.kind[kPlanes];
  c.n = n;
  c.a.assign(ctr, ctr + 3 * n);
  c.b.assign(dx, dx + n);
  c.c.assign(dy, dy + n);
  c.d.assign(rot, rot + 9 * n);
  alloc_boxes(c.boxes, n);
  const double th = std::numeric_limits<double>::min();
  for (size_t i = 0; i < n; ++i) {
    const V3 o = load3(&c.a[3 * i]);
    const double *R = &c.d[9 * i];
    const double hx = c.b[i], hy = c.c[i];
    const V3 p[6] = {o + rotate(R, {-hx / 2.0, -hy / 2.0, 0.0}),
                     o + rotate(R, {hx / 2.0, -hy / 2.0, 0.0}),
                     o + rotate(R, {-hx / 2.0, hy / 2.0, 0.0}),
                     o + rotate(R, {hx / 2.0, hy / 2.0, 0.0}),
                     o + rotate(R, {0.0, 0.0, -th}),
                     o + rotate(R, {0.0, 0.0, th})};
    six_point_box(p, &c.boxes.bmin[3 * i], &c.boxes.bmax[3 * i]);
    store3(&c.boxes.center[3 * i], o);
  }
}

// blazert/primitives/cylinder.h:115-147: box of the six points centre +- R a e_x,
// +- R b e_y, +- R (h/2) e_z (not the true box of a rotated cylinder).
void add_cylinders(HostScene &s, const double *ctr, const double *a, const double *b,
                   const double *h, const double *rot, size_t n) {
  Collection &c = s.kind[kCylinders];
  c.n = n;
  c.a.assign(ctr, ctr + 3 * n);
  c.b.assign(a, a + n);
  c.c.assign(b, b + n);
  c.d.assign(h, h + n);
  c.e.assign(rot, rot + 9 * n);
  alloc_boxes(c.boxes, n);
  for (size_t i = 0; i < n; ++i) {
    const V3 o = load3(&c.a[3 * i]);
    const double *R = &c.e[9 * i];
    const V3 ra = rotate(R, {c.b[i], 0.0, 0.0}), rb = rotate(R, {0.0, c.c[i], 0.0}),
             rh = rotate(R, {0.0, 0.0, c.d[i] / 2.0});
    const V3 p[6] = {o + ra, o + rb, o - ra, o - rb, o + rh, o - rh};
    six_point_box(p, &c.boxes.bmin[3 * i], &c.boxes.bmax[3 * i]);
    store3(&c.boxes.center[3 * i], o);
  }
}

BuildStatistics tree_statistics(const Tree &t) {
  BuildStatistics st;
  st.max_tree_depth = t.max_depth;
  st.bad_splits = t.bad_splits;
  for (const TreeNode &nd : t.nodes) {
    if (nd.leaf == 1) {
      ++st.leaf_nodes;
      st.max_num_prims_per_leaf = std::max(st.max_num_prims_per_leaf, nd.prim_cnt);
      st.min_num_prims_per_leaf = std::min(st.min_num_prims_per_leaf, nd.prim_cnt);
    } else {
      ++st.branch_nodes;
    }
  }
  return st;
}

namespace {

double box_area(const TreeNode &nd) {
  const double x = nd.mx[0] - nd.mn[0], y = nd.mx[1] - nd.mn[1], z = nd.mx[2] - nd.mn[2];
  return 2.0 * ((x * y + y * z) + z * x);
}

// Grid of one axis of a wide node: the smallest exponent e with the node's [lo, hi] covered
// by 255 cells of 2^e from k * 2^e (k = floor(lo / 2^e)) and |k|, |k + 255| below 2^24, so
// that every stored bound k' * 2^e is exact in float.  Returns false if none in [-100, 100].
bool axis_grid(double lo, double hi, int *e_out, int64_t *k_out) {
  const double m = std::max(std::abs(lo), std::abs(hi));
  int e = m > 0.0 ? std::ilogb(m) - 22 : -100;
  const double ext = hi - lo;
  if (ext > 0.0) e = std::max(e, std::ilogb(ext / 255.0) - 1);
  e = std::max(e, -100);
  for (; e <= 100; ++e) {
    const double k = std::floor(std::ldexp(lo, -e)), top = std::ceil(std::ldexp(hi, -e));
    if (top - k <= 255.0 && std::abs(k) < 16777216.0 - 256.0) {
      *e_out = e;
      *k_out = static_cast<int64_t>(k);
      return true;
    }
  }
  return false;
}

}  // namespace

// The mixed-precision image of one kind (layout.h, kWideBytes): leaf records in tree order,
// then the wide nodes breadth-first from the root's treelet.  Leaves the image's mixed_ok
// false when a box cannot be quantised or the traversal stack could exceed kLocalStack.
void build_wide(const Tree &t, int kind, const std::vector<uint32_t> &leaf_pos, KindImage *img) {
  const size_t nn = t.nodes.size();
  const uint32_t units = kind == kMesh ? 1u : uint32_t(kPayloadDoubles[kind] * 8 / 16);
  // leaf records: 4 units of header, then `units` per primitive
  std::vector<uint32_t> leaf_off(nn, 0);
  uint64_t total = 0;
  for (size_t i = 0; i < nn; ++i)
    if (t.nodes[i].leaf == 1) {
      leaf_off[i] = static_cast<uint32_t>(total);
      total += kLeafHeaderBytes / 16 + uint64_t(units) * t.nodes[i].prim_cnt;
    }
  if (total >= kIdMask) {
    img->mixed_ok = false;
    return;
  }
  img->leaves.resize(size_t(total) * 2);
  for (size_t i = 0; i < nn; ++i) {
    const TreeNode &nd = t.nodes[i];
    if (nd.leaf != 1) continue;
    double *L = &img->leaves[size_t(leaf_off[i]) * 2];
    for (int a = 0; a < 3; ++a) {
      L[2 * a] = nd.mn[a];
      L[2 * a + 1] = nd.mx[a];
    }
    const uint32_t head[4] = {leaf_pos[i], nd.prim_cnt, 0u, 0u};
    std::memcpy(L + 6, head, sizeof head);
    for (uint32_t q = 0; q < nd.prim_cnt; ++q) {
      const size_t at = size_t(leaf_pos[i]) + q;
      double *R = L + kLeafHeaderBytes / 8 + size_t(q) * units * 2;
      if (kind == kMesh) {
        const uint32_t rec[4] = {img->tri[4 * at], img->tri[4 * at + 1], img->tri[4 * at + 2], 0u};
        std::memcpy(R, rec, sizeof rec);
      } else {
        std::memcpy(R, &img->payload[at * kPayloadDoubles[kind]],
                    sizeof(double) * kPayloadDoubles[kind]);
      }
    }
  }
  img->n_leaf16 = static_cast<uint32_t>(total);
  img->n_wide = 0;
  img->wide_stack = 1;
  if (t.nodes[0].leaf == 1) {
    img->wide_root_ref = kLeafBit | leaf_off[0];
    return;
  }
  img->wide_root_ref = 0;
  // treelets, breadth-first; queue[w] is the tree node at the root of wide node w
  std::vector<uint32_t> queue{0}, depth_sum{0};
  std::vector<unsigned char> out;
  double cmax = 0.0;
  for (size_t head = 0; head < queue.size(); ++head) {
    const TreeNode &root = t.nodes[queue[head]];
    std::vector<uint32_t> ch{root.child[0], root.child[1]};
    std::vector<uint32_t> expanded{queue[head]};
    for (;;) {
      if (ch.size() >= size_t(kWideMax)) break;
      int pick = -1;
      double best = -1.0;
      for (size_t j = 0; j < ch.size(); ++j) {
        const TreeNode &c = t.nodes[ch[j]];
        if (c.leaf == 1) continue;
        const double a = box_area(c);
        if (a > best) {
          best = a;
          pick = static_cast<int>(j);
        }
      }
      if (pick < 0) break;
      const uint32_t x = ch[pick];
      expanded.push_back(x);
      ch[pick] = t.nodes[x].child[0];
      ch.insert(ch.begin() + pick + 1, t.nodes[x].child[1]);
    }
    unsigned char node[kWideBytes] = {};
    float origin[3];
    uint32_t ex = 0;
    for (int a = 0; a < 3; ++a) {
      int e = 0;
      int64_t k = 0;
      if (!axis_grid(root.mn[a], root.mx[a], &e, &k)) {
        img->mixed_ok = false;
        return;
      }
      origin[a] = static_cast<float>(std::ldexp(static_cast<double>(k), e));
      cmax = std::max({cmax, std::abs(std::ldexp(static_cast<double>(k), e)),
                       std::abs(std::ldexp(static_cast<double>(k + 255), e))});
      ex |= uint32_t(e + 127) << (8 * a);
      for (size_t j = 0; j < size_t(kWideMax); ++j) {
        unsigned char lo = 255, hi = 0;
        if (j < ch.size()) {
          const TreeNode &c = t.nodes[ch[j]];
          const double ql = std::floor(std::ldexp(c.mn[a], -e)) - static_cast<double>(k);
          const double qh = std::ceil(std::ldexp(c.mx[a], -e)) - static_cast<double>(k);
          if (!(ql >= 0.0 && qh <= 255.0 && ql <= qh)) {
            img->mixed_ok = false;
            return;
          }
          lo = static_cast<unsigned char>(ql);
          hi = static_cast<unsigned char>(qh);
        }
        node[16 + 16 * a + j] = lo;
        node[24 + 16 * a + j] = hi;
      }
    }
    ex |= uint32_t(ch.size()) << 24;
    std::memcpy(node, origin, sizeof origin);
    std::memcpy(node + 12, &ex, sizeof ex);
    // perm nibbles past the children hold 15: no slot, so the walk never takes them
    uint32_t ref[kWideMax] = {}, perm[8] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu,
                                            0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
    for (size_t j = 0; j < ch.size(); ++j) {
      const TreeNode &c = t.nodes[ch[j]];
      if (c.leaf == 1) {
        ref[j] = kLeafBit | leaf_off[ch[j]];
      } else {
        ref[j] = static_cast<uint32_t>(queue.size());
        queue.push_back(ch[j]);
        depth_sum.push_back(depth_sum[head] + uint32_t(ch.size()) - 1);
      }
    }
    // visit order per octant: at every expanded node the child on the ray's sign side first
    for (uint32_t oct = 0; oct < 8; ++oct) {
      uint32_t pos = 0;
      std::vector<uint32_t> todo{queue[head]};
      while (!todo.empty()) {
        const uint32_t x = todo.back();
        todo.pop_back();
        const auto it = std::find(ch.begin(), ch.end(), x);
        if (it != ch.end() && x != queue[head]) {
          perm[oct] &= ~(0xFu << (4 * pos));
          perm[oct] |= uint32_t(it - ch.begin()) << (4 * pos++);
          continue;
        }
        const TreeNode &nx = t.nodes[x];
        const uint32_t first = (oct >> nx.axis) & 1u;
        todo.push_back(nx.child[1 - first]);
        todo.push_back(nx.child[first]);
      }
    }
    std::memcpy(node + 64, ref, sizeof ref);
    std::memcpy(node + 96, perm, sizeof perm);
    out.insert(out.end(), node, node + kWideBytes);
    img->wide_stack = std::max(img->wide_stack, depth_sum[head] + uint32_t(ch.size()) - 1);
  }
  if (img->wide_stack > kLocalStack || !(cmax <= 1e18)) {
    img->mixed_ok = false;
    return;
  }
  img->n_wide = static_cast<uint32_t>(queue.size());
  img->wide.assign(out.begin(), out.end());
  img->wide_coord_max = round_up(cmax);
}

KindImage flatten(const HostScene &s, int kind, size_t max_workers) {
  const Collection &c = s.kind[kind];
  const Tree &t = c.tree;
  KindImage img;
  const size_t nn = t.nodes.size();
  // Leaf positions in the leaf-ordered primitive arrays follow the tree's node order.
  std::vector<uint32_t> leaf_pos(nn, 0), dev_index(nn, 0xFFFFFFFFu);
  uint32_t pos = 0;
  for (size_t i = 0; i < nn; ++i)
    if (t.nodes[i].leaf == 1) {
      leaf_pos[i] = pos;
      pos += t.nodes[i].prim_cnt;
    }
  // Breadth-first numbering of the internal nodes; the order array is its own FIFO queue.
  std::vector<uint32_t> order;
  if (nn && t.nodes[0].leaf != 1) {
    order.reserve(nn / 2 + 1);
    order.push_back(0);
    for (size_t head = 0; head < order.size(); ++head) {
      const uint32_t i = order[head];
      dev_index[i] = static_cast<uint32_t>(head);
      for (int j = 0; j < 2; ++j) {
        const uint32_t ch = t.nodes[i].child[j];
        if (t.nodes[ch].leaf != 1) order.push_back(ch);
      }
    }
  }
  auto ref_of = [&](uint32_t i) {
    return t.nodes[i].leaf == 1 ? (kLeafBit | leaf_pos[i]) : dev_index[i];
  };
  auto finite_box = [](const TreeNode &nd) {
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(nd.mn[k]) || !std::isfinite(nd.mx[k])) return false;
    return true;
  };
  img.n_internal = static_cast<uint32_t>(order.size());
  img.nodes64.resize(size_t(img.n_internal) * kNode64Doubles);
  // Each node reads only the tree and writes only its own slots, so ranges of nodes can be
  // filled on separate threads.
  const size_t workers =
      range_workers(img.n_internal, kNodesPerRange, max_workers);
  std::vector<char> finite(workers, 1);
  run_ranges(img.n_internal, workers, [&](size_t g0, size_t g1, size_t w) {
    for (size_t g = g0; g < g1; ++g) {
      const TreeNode &nd = t.nodes[order[g]];
      double *d = &img.nodes64[g * kNode64Doubles];
      for (int j = 0; j < 2; ++j) {
        const TreeNode &ch = t.nodes[nd.child[j]];
        if (!finite_box(ch)) finite[w] = 0;
        for (int k = 0; k < 3; ++k) {
          d[6 * j + 2 * k] = ch.mn[k];
          d[6 * j + 2 * k + 1] = ch.mx[k];
        }
      }
      const uint32_t meta[4] = {ref_of(nd.child[0]), ref_of(nd.child[1]), nd.axis, 0u};
      std::memcpy(d + 12, meta, sizeof meta);
      d[14] = d[15] = 0.0;
    }
  });
  for (const char ok : finite)
    if (!ok) img.mixed_ok = false;
  if (nn) {
    const TreeNode &root = t.nodes[0];
    img.root_ref = ref_of(0);
    if (!finite_box(root)) img.mixed_ok = false;
    double cmax = 0.0;
    for (int k = 0; k < 3; ++k) {
      img.root_box[2 * k] = root.mn[k];
      img.root_box[2 * k + 1] = root.mx[k];
      cmax = std::max(cmax, std::max(std::abs(root.mn[k]), std::abs(root.mx[k])));
    }
    img.coord_max = round_up(cmax);
    if (!(cmax <= 1e18)) img.mixed_ok = false;
  }
  // Leaf-ordered primitives: leaves own disjoint position ranges and the ids are a
  // permutation, so ranges of leaves can be written on separate threads.
  const size_t np = t.leaf_prims.size();
  const int stride = kPayloadDoubles[kind];
  img.prim_ids.resize(np);
  img.pos_of.assign(np, 0u);
  img.payload.assign(np * stride, 0.0);
  run_ranges(nn, range_workers(nn, kNodesPerRange, max_workers),
             [&](size_t i0, size_t i1, size_t) {
    for (size_t i = i0; i < i1; ++i) {
      const TreeNode &nd = t.nodes[i];
      if (nd.leaf != 1) continue;
      for (uint32_t q = 0; q < nd.prim_cnt; ++q) {
        const uint32_t at = leaf_pos[i] + q;
        const uint32_t id = t.leaf_prims[nd.prim_off + q];
        img.prim_ids[at] = id | (q + 1 == nd.prim_cnt ? kLastBit : 0u);
        img.pos_of[id] = at;
        double *p = img.payload.data() + size_t(at) * stride;
        switch (kind) {
          case kSpheres:
            for (int k = 0; k < 3; ++k) p[k] = c.a[3 * id + k];
            p[3] = c.b[id];
            break;
          case kPlanes:
            for (int k = 0; k < 3; ++k) p[k] = c.a[3 * id + k];
            p[3] = c.b[id];
            p[4] = c.c[id];
            for (int k = 0; k < 9; ++k) p[5 + k] = c.d[9 * id + k];
            break;
          case kCylinders:
            for (int k = 0; k < 3; ++k) p[k] = c.a[3 * id + k];
            p[3] = c.b[id];
            p[4] = c.c[id];
            p[5] = c.d[id];
            for (int k = 0; k < 9; ++k) p[6 + k] = c.e[9 * id + k];
            break;
          default:
            break;
        }
      }
    }
  });
  if (kind == kMesh)
    number_vertices(s, &img, range_workers(np, kPrimsPerRange, max_workers));
  // Cylinders may move the hit distance outward (blazert/primitives/cylinder.h:181-495), which
  // the wide image's exactness argument excludes; their mixed mode runs the FP64 traversal.
  if (img.mixed_ok && kind != kCylinders && nn) build_wide(t, kind, leaf_pos, &img);
  else img.mixed_ok = false;
  return img;
}

}  // namespace bzr
