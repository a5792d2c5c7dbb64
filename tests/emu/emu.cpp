// CPU emulator of the GPU traversal (TEST INFRASTRUCTURE ONLY, never linked into the product).
//
// Compiles the kernels' own per-ray code (blazert_b200/csrc/trace_core.cuh) and the product's
// host builder and flattener (scene.cpp) as host code, so that the tests can check the device
// layout and the deferred-key traversal against the oracle on machines without a GPU.
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../blazert_b200/csrc/layout.h"
#include "../../blazert_b200/csrc/scene.h"
#include "../../blazert_b200/csrc/trace_core.cuh"
#include "../../blazert_b200/csrc/distance_core.cuh"

namespace {
struct Emu {
  bzr::HostScene host;
  std::vector<bzr::KindImage> img;
  bzr::SceneView view;
};
}  // namespace

// Builds (or, for a loaded scene, keeps) every kind's tree, flattens it and fills the view.
static void commit(Emu *e, bool build) {
  bzr::HostScene &s = e->host;
  e->img.resize(4);
  uint32_t depth = 0;
  for (int k = 0; k < 4; ++k) {
    bzr::Collection &c = s.kind[k];
    bzr::KindView &v = e->view.k[k];
    v.present = c.present;
    v.geom_id = c.geom_id;
    if (!c.present) continue;
    if (build) c.tree = bzr::build_tree(c.boxes, s.opt);
    depth = depth > c.tree.max_depth ? depth : c.tree.max_depth;
    e->img[k] = bzr::flatten(s, k);
    const bzr::KindImage &im = e->img[k];
    v.nodes64 = im.nodes64.data();
    v.wide = im.wide.data();
    v.leaves = im.leaves.data();
    v.n_wide = im.n_wide;
    v.n_leaf16 = im.n_leaf16;
    v.wide_root_ref = im.wide_root_ref;
    v.payload = im.payload.data();
    v.prim_ids = im.prim_ids.data();
    v.pos_of = im.pos_of.data();
    v.tri = im.tri.data();
    v.verts = im.verts.data();
    v.vnorm = im.vnorm.data();
    v.n_internal = im.n_internal;
    v.n_prims = static_cast<uint32_t>(im.prim_ids.size());
    v.n_verts = static_cast<uint32_t>(im.verts.size() / bzr::kVertexDoubles);
    v.root_ref = im.root_ref;
    v.mixed_ok = im.mixed_ok;
    std::memcpy(v.root_box, im.root_box, sizeof v.root_box);
    v.coord_max = im.coord_max;
  }
  e->view.faces = s.faces.data();
  e->view.vert_n = s.vert_n.data();
  uint32_t cap = (depth + 2) < 8 ? 8 : depth + 2;
  for (int k = 0; k < 4; ++k)
    if (s.kind[k].present && e->img[k].mixed_ok && e->img[k].wide_stack > cap)
      cap = e->img[k].wide_stack;
  e->view.stack_cap = cap;
  s.committed = true;
}


extern "C" {

void *emu_scene_create(const int *order, int n_order, const double *verts, long n_verts,
                 const uint32_t *faces, long n_faces, const double *sph_c, const double *sph_r,
                 long n_sph, const double *pl_c, const double *pl_dx, const double *pl_dy,
                 const double *pl_rot, long n_pl, const double *cy_c, const double *cy_a,
                 const double *cy_b, const double *cy_h, const double *cy_rot, long n_cy,
                 unsigned min_leaf, unsigned max_depth, unsigned bins, uint32_t *geom_ids) {
  auto *e = new Emu();
  bzr::HostScene &s = e->host;
  for (int j = 0; j < n_order; ++j) {
    const int k = order[j];
    uint32_t id = 0xFFFFFFFFu;
    if (k >= 0 && k < 4 && !s.kind[k].present) {
      switch (k) {
        case 0: bzr::add_mesh(s, verts, n_verts, faces, n_faces); break;
        case 1: bzr::add_spheres(s, sph_c, sph_r, n_sph); break;
        case 2: bzr::add_planes(s, pl_c, pl_dx, pl_dy, pl_rot, n_pl); break;
        case 3: bzr::add_cylinders(s, cy_c, cy_a, cy_b, cy_h, cy_rot, n_cy); break;
      }
      s.kind[k].present = true;
      id = s.kind[k].geom_id = s.geometries++;
    }
    if (geom_ids) geom_ids[j] = id;
  }
  s.opt.min_leaf = min_leaf;
  s.opt.max_depth = max_depth;
  s.opt.bins = bins;
  commit(e, true);
  return e;
}

// The persistent scene format (scene_io.cpp) on the CPU: bytes of a scene, and a scene from
// bytes (NULL and the reason in `why` when they are refused).
long emu_scene_encode(void *h, uint8_t *out, long cap) {
  const auto b = bzr::encode_scene(static_cast<Emu *>(h)->host);
  if (out && cap >= static_cast<long>(b.size())) std::memcpy(out, b.data(), b.size());
  return static_cast<long>(b.size());
}

void *emu_scene_decode(const uint8_t *data, long size, char *why, long why_cap) {
  auto *e = new Emu();
  const std::string err = bzr::decode_scene(data, static_cast<size_t>(size), &e->host);
  if (!err.empty()) {
    if (why && why_cap > 0) {
      std::strncpy(why, err.c_str(), static_cast<size_t>(why_cap) - 1);
      why[why_cap - 1] = 0;
    }
    delete e;
    return nullptr;
  }
  commit(e, false);
  return e;
}

void emu_scene_destroy(void *h) { delete static_cast<Emu *>(h); }

// Same dump layout as the oracle's ora_scene_tree.
long emu_scene_tree(void *h, int kind, double *bmin, double *bmax, uint32_t *leaf, uint32_t *axis,
              uint32_t *children, uint32_t *prim_off, uint32_t *prim_cnt, uint32_t *prim_ids,
              long prim_cap) {
  const Emu *e = static_cast<Emu *>(h);
  if (kind < 0 || kind > 3 || !e->host.kind[kind].present) return -1;
  const bzr::Tree &t = e->host.kind[kind].tree;
  const long n = static_cast<long>(t.nodes.size());
  if (!bmin) return n;
  uint32_t running = 0;
  for (long i = 0; i < n; ++i) {
    const bzr::TreeNode &nd = t.nodes[i];
    std::memcpy(bmin + 3 * i, nd.mn, 24);
    std::memcpy(bmax + 3 * i, nd.mx, 24);
    leaf[i] = nd.leaf;
    axis[i] = nd.axis;
    children[2 * i] = nd.child[0];
    children[2 * i + 1] = nd.child[1];
    prim_off[i] = running;
    prim_cnt[i] = nd.leaf == 1 ? nd.prim_cnt : 0;
    running += prim_cnt[i];
  }
  for (long i = 0; i < static_cast<long>(t.leaf_prims.size()) && i < prim_cap; ++i)
    prim_ids[i] = t.leaf_prims[i];
  return n;
}

// Runs the kernels' per-ray code with the kernels' data flow: one pass per kind present, in the
// reference's kind order, each merged into the output arrays by finalize_kind.  Returns the
// accumulated error word.
}  // extern "C"

// Work counters of one kind over a batch (the kernels' Counts, summed): totals[16] as
// bzr_work_counts_ex lays them out (box, prim, node, leaf; each per kind).
template <int KIND>
static void emu_count_pass(const bzr::SceneView &view, long n, const double *org,
                           const double *dir, const double *tmin, const double *tmax, int mode,
                           uint64_t *totals) {
  uint64_t box = 0, prim = 0, node = 0, leaf = 0;
#pragma omp parallel reduction(+ : box, prim, node, leaf)
  {
    std::vector<double> key(view.stack_cap);
    std::vector<uint32_t> ref(view.stack_cap);
    bzr::Stack sk;
    sk.key = key.data();
    sk.ref = ref.data();
    sk.cap = view.stack_cap;
    sk.stride = 1;
    uint32_t e = 0;
#pragma omp for schedule(dynamic, 256)
    for (long i = 0; i < n; ++i) {
      bzr::Ray r = bzr::make_ray(org + 3 * i, dir + 3 * i, tmin ? tmin[i] : 0.0,
                                 tmax ? tmax[i] : 1.7976931348623157e308);
      bzr::KState st;
      bzr::Counts c = {};
      if (mode & 1)
        bzr::traverse_mixed<KIND, true>(view.k[KIND], r, st, sk, 0, &e, &c);
      else
        bzr::traverse<KIND, true>(view.k[KIND], r, st, sk, 0, &e, &c);
      box += c.box[KIND];
      prim += c.prim[KIND];
      node += c.node[KIND];
      leaf += c.leaf[KIND];
    }
  }
  totals[KIND] += box;
  totals[4 + KIND] += prim;
  totals[8 + KIND] += node;
  totals[12 + KIND] += leaf;
}

template <int KIND>
static void emu_pass(const bzr::SceneView &view, long n, const double *org, const double *dir,
                     const double *tmin, const double *tmax, bool first, double *t, double *uv,
                     double *normal, uint32_t *prim, uint32_t *geom, uint8_t *hit, uint32_t &err,
                     int mode) {
  uint32_t e = 0;
#pragma omp parallel reduction(| : e)
  {
    std::vector<double> key(view.stack_cap);
    std::vector<uint32_t> ref(view.stack_cap);
    bzr::Stack sk;
    sk.key = key.data();
    sk.ref = ref.data();
    sk.cap = view.stack_cap;
    sk.stride = 1;
#pragma omp for schedule(dynamic, 256)
    for (long i = 0; i < n; ++i) {
      bzr::Ray r = bzr::make_ray(org + 3 * i, dir + 3 * i, tmin ? tmin[i] : 0.0,
                                 tmax ? tmax[i] : 1.7976931348623157e308);
      r.any_hit = (mode & 2) != 0;
      bzr::KState st;
      if (mode & 1)
        bzr::traverse_mixed<KIND, false>(view.k[KIND], r, st, sk, 0, &e, nullptr);
      else
        bzr::traverse<KIND, false>(view.k[KIND], r, st, sk, 0, &e, nullptr);
      bzr::finalize_kind<KIND>(view, r, st, uint64_t(i), first, t, uv, normal, prim, geom, hit);
    }
  }
  err |= e;
}

extern "C" {

// Checks one kind's wide image against its tree: every leaf record is reached exactly once
// from the wide root, every stored child box on the way contains the leaf's exact box (the
// bounds origin + q 2^e evaluated exactly in double), and every leaf record's box and
// primitive range are the tree leaf's.  Returns the number of violations, or -1 when the kind
// has no wide image; *leaves receives the leaf records reached.
long emu_wide_check(void *h, int kind, long *leaves) {
  const Emu *e = static_cast<Emu *>(h);
  const bzr::KindImage &im = e->img[kind];
  *leaves = 0;
  if (!e->host.kind[kind].present || !im.mixed_ok) return -1;
  long bad = 0;
  std::vector<long> seen(im.n_leaf16, 0);
  struct Box {
    double lo[3], hi[3];
  };
  struct Item {
    uint32_t ref;
    std::vector<Box> path;
  };
  std::vector<Item> todo{{im.wide_root_ref, {}}};
  while (!todo.empty()) {
    Item it = todo.back();
    todo.pop_back();
    if (it.ref & bzr::kLeafBit) {
      const uint32_t off = it.ref & bzr::kIdMask;
      if (off >= im.n_leaf16) {
        ++bad;
        continue;
      }
      ++seen[off];
      ++*leaves;
      const double *L = &im.leaves[2 * size_t(off)];
      for (const Box &b : it.path)
        for (int a = 0; a < 3; ++a)
          if (!(b.lo[a] <= L[2 * a] && L[2 * a + 1] <= b.hi[a])) ++bad;
      continue;
    }
    if (it.ref >= im.n_wide) {
      ++bad;
      continue;
    }
    const unsigned char *nd = &im.wide[size_t(it.ref) * bzr::kWideBytes];
    float origin[3];
    uint32_t ex, refs[8];
    std::memcpy(origin, nd, 12);
    std::memcpy(&ex, nd + 12, 4);
    std::memcpy(refs, nd + 64, 32);
    const uint32_t nch = ex >> 24;
    if (nch < 2 || nch > 8) ++bad;
    for (uint32_t c = 0; c < nch && c < 8; ++c) {
      Item child{refs[c], it.path};
      Box b;
      for (int a = 0; a < 3; ++a) {
        const int ea = int((ex >> (8 * a)) & 0xFFu) - 127;
        b.lo[a] = double(origin[a]) + std::ldexp(double(nd[16 + 16 * a + c]), ea);
        b.hi[a] = double(origin[a]) + std::ldexp(double(nd[24 + 16 * a + c]), ea);
      }
      child.path.push_back(b);
      todo.push_back(child);
    }
  }
  // every leaf of the tree has its record (records are in tree order), with its box and
  // primitive range, reached once
  const bzr::Tree &t = e->host.kind[kind].tree;
  long n_leaves = 0;
  for (const bzr::TreeNode &nd : t.nodes) n_leaves += nd.leaf == 1 ? 1 : 0;
  if (n_leaves != *leaves) ++bad;
  size_t off = 0;
  uint32_t first = 0;
  const uint32_t units = kind == 0 ? 1u : uint32_t(bzr::kPayloadDoubles[kind] / 2);
  for (const bzr::TreeNode &nd : t.nodes) {
    if (nd.leaf != 1) continue;
    if (off + 4 > im.n_leaf16 || seen[off] != 1) {
      ++bad;
      break;
    }
    const double *L = &im.leaves[2 * off];
    uint32_t head[2];
    std::memcpy(head, L + 6, 8);
    for (int a = 0; a < 3; ++a)
      if (L[2 * a] != nd.mn[a] || L[2 * a + 1] != nd.mx[a]) ++bad;
    if (head[0] != first || head[1] != nd.prim_cnt) ++bad;
    first += nd.prim_cnt;
    off += 4 + size_t(units) * nd.prim_cnt;
  }
  return bad;
}

void emu_work_counts(void *h, long n, const double *org, const double *dir, const double *tmin,
                     const double *tmax, int mode, uint64_t *totals) {
  const Emu *e = static_cast<Emu *>(h);
  for (int k = 0; k < 16; ++k) totals[k] = 0;
  for (int k = 0; k < 4; ++k) {
    if (!e->view.k[k].present || e->view.k[k].n_prims == 0) continue;
    switch (k) {
      case 0: emu_count_pass<0>(e->view, n, org, dir, tmin, tmax, mode, totals); break;
      case 1: emu_count_pass<1>(e->view, n, org, dir, tmin, tmax, mode, totals); break;
      case 2: emu_count_pass<2>(e->view, n, org, dir, tmin, tmax, mode, totals); break;
      default: emu_count_pass<3>(e->view, n, org, dir, tmin, tmax, mode, totals); break;
    }
  }
}

uint32_t emu_scene_intersect(void *h, long n, const double *org, const double *dir,
                             const double *tmin, const double *tmax, double *t, double *uv,
                             double *normal, uint32_t *prim, uint32_t *geom, uint8_t *hit,
                             uint32_t stack_cap_override, int mode) {
  const Emu *e = static_cast<Emu *>(h);
  bzr::SceneView view = e->view;
  if (stack_cap_override) view.stack_cap = stack_cap_override;
  uint32_t err = 0;
  bool first = true;
  for (int k = 0; k < 4; ++k) {
    if (!view.k[k].present || view.k[k].n_prims == 0) continue;
    switch (k) {
      case 0: emu_pass<0>(view, n, org, dir, tmin, tmax, first, t, uv, normal, prim, geom, hit, err, mode); break;
      case 1: emu_pass<1>(view, n, org, dir, tmin, tmax, first, t, uv, normal, prim, geom, hit, err, mode); break;
      case 2: emu_pass<2>(view, n, org, dir, tmin, tmax, first, t, uv, normal, prim, geom, hit, err, mode); break;
      case 3: emu_pass<3>(view, n, org, dir, tmin, tmax, first, t, uv, normal, prim, geom, hit, err, mode); break;
    }
    first = false;
  }
  if (first)
    for (long i = 0; i < n; ++i) {
      t[i] = 1.7976931348623157e308;
      uv[2 * i] = uv[2 * i + 1] = 0.0;
      normal[3 * i] = normal[3 * i + 1] = normal[3 * i + 2] = 0.0;
      prim[i] = geom[i] = 0xFFFFFFFFu;
      hit[i] = 0;
    }
  return err;
}

// Precomputed box and centre of one primitive (the product's collection precompute).
int emu_prim_box(void *h, int kind, uint32_t id, double *mn, double *mx, double *center) {
  const Emu *e = static_cast<Emu *>(h);
  if (kind < 0 || kind > 3 || !e->host.kind[kind].present || id >= e->host.kind[kind].n) return -1;
  const bzr::PrimBoxes &b = e->host.kind[kind].boxes;
  std::memcpy(mn, &b.bmin[3 * size_t(id)], 24);
  std::memcpy(mx, &b.bmax[3 * size_t(id)], 24);
  std::memcpy(center, &b.center[3 * size_t(id)], 24);
  return 0;
}

// The kernels' slab test of one box, decided for the hit distance `tmax` as at pop time:
// returns 1 when the reference's intersect_node(tmin, tmax, box, ray) would accept the box.
int emu_box_accept(const double *bmin, const double *bmax, const double *org, const double *dir,
                   double tmin, double tmax) {
  const bzr::Ray r = bzr::make_ray(org, dir, tmin, tmax);
  double key;
  const bool p = bzr::box_test(make_double2(bmin[0], bmax[0]), make_double2(bmin[1], bmax[1]),
                               make_double2(bmin[2], bmax[2]), r, key);
  return (p && !(key > tmax)) ? 1 : 0;
}

// The distance kernels' per-point code (distance_core.cuh): per-primitive form and the
// scene-level nearest surface with its BVH pruning.  Returns the error bits.
uint32_t emu_distance_to_surface(void *h, int kind, long n, const uint32_t *ids,
                                 const double *points, double *distance, double *closest) {
  const Emu *e = static_cast<Emu *>(h);
  uint32_t err = 0;
  for (long i = 0; i < n; ++i) {
    bzr::D3 c;
    bool bad = false;
    const bzr::D3 p = bzr::d3(points[3 * i], points[3 * i + 1], points[3 * i + 2]);
    distance[i] = bzr::distance_query(e->view, kind, ids[i], p, &c, &bad);
    if (closest) {
      closest[3 * i] = c.x;
      closest[3 * i + 1] = c.y;
      closest[3 * i + 2] = c.z;
    }
    if (bad) err |= bzr::kErrPrimIndex;
  }
  return err;
}

void emu_closest_surface(void *h, long n, const double *points, double *distance, uint32_t *prim,
                         uint32_t *geom) {
  const Emu *e = static_cast<Emu *>(h);
  uint32_t stack_ref[64];
  float stack_key[64];
  for (long i = 0; i < n; ++i) {
    const bzr::D3 p = bzr::d3(points[3 * i], points[3 * i + 1], points[3 * i + 2]);
    const bzr::NearestState st = bzr::nearest_surface(e->view, p, stack_ref, stack_key, 64);
    distance[i] = st.best;
    if (prim) prim[i] = st.prim;
    if (geom) geom[i] = st.geom;
  }
}

// The product's OBJ reader (obj.cpp), for the sanitizer run: vertices and faces into the
// caller's arrays (when large enough); returns 0, or 1 with the reason in `why`.
int emu_obj_load(const char *path, double *v, long vcap, uint32_t *f, long fcap, long *nv,
                 long *nf, char *why, long why_cap) {
  std::vector<double> vv;
  std::vector<uint32_t> ff;
  const std::string err = bzr::load_obj(path, &vv, &ff);
  if (!err.empty()) {
    if (why && why_cap > 0) {
      std::strncpy(why, err.c_str(), static_cast<size_t>(why_cap) - 1);
      why[why_cap - 1] = 0;
    }
    return 1;
  }
  *nv = static_cast<long>(vv.size() / 3);
  *nf = static_cast<long>(ff.size() / 3);
  if (v && vcap >= static_cast<long>(vv.size())) std::memcpy(v, vv.data(), vv.size() * 8);
  if (f && fcap >= static_cast<long>(ff.size())) std::memcpy(f, ff.data(), ff.size() * 4);
  return 0;
}

// The build statistics of one kind's tree (host builder): max depth, leaf nodes, max and
// min primitives per leaf, branch nodes, bad splits.  Returns -1 for an absent kind.
int emu_build_statistics(void *h, int kind, uint32_t *out) {
  const bzr::Collection &c = static_cast<Emu *>(h)->host.kind[kind];
  if (!c.present) return -1;
  const bzr::BuildStatistics st = bzr::tree_statistics(c.tree);
  const uint32_t v[6] = {st.max_tree_depth, st.leaf_nodes, st.max_num_prims_per_leaf,
                         st.min_num_prims_per_leaf, st.branch_nodes, st.bad_splits};
  std::memcpy(out, v, sizeof v);
  return 0;
}

// FNV-1a digest of every array and field of one kind's device image, flattened again with at
// most `workers` threads.  Returns -1 for an absent kind.
int emu_image_digest(void *h, int kind, long workers, uint64_t *digest) {
  const bzr::HostScene &s = static_cast<Emu *>(h)->host;
  if (!s.kind[kind].present) return -1;
  const bzr::KindImage im = bzr::flatten(s, kind, static_cast<size_t>(workers));
  uint64_t x = 1469598103934665603ull;
  auto mix = [&](const void *p, size_t n) {
    const auto *b = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < n; ++i) x = (x ^ b[i]) * 1099511628211ull;
  };
  auto mix_array = [&](const auto &v) {
    const uint64_t n = v.size();
    mix(&n, sizeof n);
    mix(v.data(), v.size() * sizeof v[0]);
  };
  mix_array(im.nodes64);
  mix_array(im.wide);
  mix_array(im.leaves);
  mix_array(im.payload);
  mix_array(im.prim_ids);
  mix_array(im.pos_of);
  mix_array(im.tri);
  mix_array(im.verts);
  mix_array(im.vnorm);
  const uint8_t ok = im.mixed_ok;
  mix(&im.n_internal, sizeof im.n_internal);
  mix(&im.root_ref, sizeof im.root_ref);
  mix(im.root_box, sizeof im.root_box);
  mix(&im.coord_max, sizeof im.coord_max);
  mix(&im.n_wide, sizeof im.n_wide);
  mix(&im.n_leaf16, sizeof im.n_leaf16);
  mix(&im.wide_root_ref, sizeof im.wide_root_ref);
  mix(&im.wide_stack, sizeof im.wide_stack);
  mix(&im.wide_coord_max, sizeof im.wide_coord_max);
  mix(&ok, 1);
  *digest = x;
  return 0;
}

}  // extern "C"
