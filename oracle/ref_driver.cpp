// C-ABI driver around the UNMODIFIED blazeRT headers (test infrastructure, not product code).
//
// oracle/Makefile compiles this file against the reference's own headers (blazert/scene.h and
// everything it includes) and the blaze-API shim in oracle/shim/, writing the result to
// oracle/_ref/.  It is used
//   * by the tests, to pin the C restatement (oracle/bzr_oracle.c) and the CUDA path against the
//     reference's own traversal and BVH build, and
//   * by bench.py's CPU-baseline leg, as the reference's intersect1 loop parallelised with OpenMP
//     over rows of 512 rays (the pattern of examples/scene_primitives/main.cc:86-110).
//
// Everything that computes lives in the reference headers; this file only converts plain arrays
// into the reference's containers (blazert/scene.h:227-346 keeps const& to them, so they are
// owned here) and copies RayHit fields out (blazert/ray.h:72-85).
#include <blazert/blazert.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

using namespace blazert;

namespace {

struct RefScene {
  Vec3rList<double> verts;
  Vec3iList faces;
  Vec3rList<double> sph_c;
  std::vector<double> sph_r;
  Vec3rList<double> pl_c;
  std::vector<double> pl_dx, pl_dy;
  Mat3rList<double> pl_rot;
  Vec3rList<double> cy_c;
  std::vector<double> cy_a, cy_b, cy_h;
  Mat3rList<double> cy_rot;
  std::unique_ptr<BlazertScene<double>> scene;
  double commit_seconds = 0.0;
};

Vec3r<double> v3(const double *p) { return Vec3r<double>{p[0], p[1], p[2]}; }
Mat3r<double> m3(const double *p) {
  Mat3r<double> m;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m(i, j) = p[3 * i + j];
  return m;
}

template <template <typename> class C>
const BVH<double, C> *bvh_of(const RefScene *s);
template <>
const BVH<double, TriangleMesh> *bvh_of<TriangleMesh>(const RefScene *s) {
  return s->scene->has_triangles ? s->scene->triangles_bvh.get() : nullptr;
}
template <>
const BVH<double, SphereCollection> *bvh_of<SphereCollection>(const RefScene *s) {
  return s->scene->has_spheres ? s->scene->spheres_bvh.get() : nullptr;
}
template <>
const BVH<double, PlaneCollection> *bvh_of<PlaneCollection>(const RefScene *s) {
  return s->scene->has_planes ? s->scene->planes_bvh.get() : nullptr;
}
template <>
const BVH<double, CylinderCollection> *bvh_of<CylinderCollection>(const RefScene *s) {
  return s->scene->has_cylinders ? s->scene->cylinders_bvh.get() : nullptr;
}

// Node dump: per node min[3], max[3], leaf, axis, children[2]; leaf primitives are appended to
// prim_ids in node order, with prim_off[node] / prim_cnt[node] locating them.
template <template <typename> class C>
long dump_tree(const RefScene *s, double *bmin, double *bmax, uint32_t *leaf, uint32_t *axis,
               uint32_t *children, uint32_t *prim_off, uint32_t *prim_cnt, uint32_t *prim_ids,
               long prim_cap) {
  const BVH<double, C> *bvh = bvh_of<C>(s);
  if (!bvh) return -1;
  long p = 0;
  const long n = static_cast<long>(bvh->nodes.size());
  if (!bmin) return n;
  for (long i = 0; i < n; ++i) {
    const auto &node = bvh->nodes[i];
    for (int k = 0; k < 3; ++k) {
      bmin[3 * i + k] = node.min[k];
      bmax[3 * i + k] = node.max[k];
    }
    leaf[i] = node.leaf;
    axis[i] = node.axis;
    children[2 * i] = node.children[0];
    children[2 * i + 1] = node.children[1];
    prim_off[i] = static_cast<uint32_t>(p);
    prim_cnt[i] = static_cast<uint32_t>(node.primitives.size());
    for (const auto &prim : node.primitives) {
      if (p < prim_cap) prim_ids[p] = prim.prim_id;
      ++p;
    }
  }
  return n;
}

// The reference's own BVHBuildStatistics (blazert/bvh/statistics.h:11-38) of one kind: a fresh
// BVH over the scene's collection built by SAHBinnedBuilder with the scene's options (the
// statistics Scene::commit drops).  out: max_tree_depth, leaf_nodes, max_num_prims_per_leaf,
// min_num_prims_per_leaf, branch_nodes, bad_splits.  Returns -1 for an absent kind.
template <template <typename> class C>
int build_statistics(const RefScene *s, uint32_t *out) {
  const BVH<double, C> *have = bvh_of<C>(s);
  if (!have) return -1;
  BVH<double, C> bvh(have->collection);
  SAHBinnedBuilder builder;
  const auto st = builder.build(bvh, s->scene->build_options);
  const uint32_t v[6] = {st.max_tree_depth, st.leaf_nodes, st.max_num_prims_per_leaf,
                         st.min_num_prims_per_leaf, st.branch_nodes, st.bad_splits};
  std::memcpy(out, v, sizeof v);
  return 0;
}

}  // namespace

extern "C" {

// kinds: 0 mesh, 1 spheres, 2 planes, 3 cylinders.  order[] lists the kinds in add order
// (the order decides geom ids, blazert/scene.h:235); n_order entries.
void *ref_scene_create(const int *order, int n_order, const double *verts, long n_verts,
                       const uint32_t *faces, long n_faces, const double *sph_c, const double *sph_r,
                       long n_sph, const double *pl_c, const double *pl_dx, const double *pl_dy,
                       const double *pl_rot, long n_pl, const double *cy_c, const double *cy_a,
                       const double *cy_b, const double *cy_h, const double *cy_rot, long n_cy,
                       unsigned min_leaf, unsigned max_depth, unsigned bins, uint32_t *geom_ids) {
  auto *s = new RefScene();
  for (long i = 0; i < n_verts; ++i) s->verts.push_back(v3(verts + 3 * i));
  for (long i = 0; i < n_faces; ++i)
    s->faces.push_back(Vec3ui{faces[3 * i], faces[3 * i + 1], faces[3 * i + 2]});
  for (long i = 0; i < n_sph; ++i) {
    s->sph_c.push_back(v3(sph_c + 3 * i));
    s->sph_r.push_back(sph_r[i]);
  }
  for (long i = 0; i < n_pl; ++i) {
    s->pl_c.push_back(v3(pl_c + 3 * i));
    s->pl_dx.push_back(pl_dx[i]);
    s->pl_dy.push_back(pl_dy[i]);
    s->pl_rot.push_back(m3(pl_rot + 9 * i));
  }
  for (long i = 0; i < n_cy; ++i) {
    s->cy_c.push_back(v3(cy_c + 3 * i));
    s->cy_a.push_back(cy_a[i]);
    s->cy_b.push_back(cy_b[i]);
    s->cy_h.push_back(cy_h[i]);
    s->cy_rot.push_back(m3(cy_rot + 9 * i));
  }
  s->scene = std::make_unique<BlazertScene<double>>();
  // BVHBuildOptions has const members (blazert/bvh/options.h:16-18): rebuild it in place.
  s->scene->build_options.~BVHBuildOptions<double>();
  new (&s->scene->build_options) BVHBuildOptions<double>(min_leaf, max_depth, bins);
  for (int k = 0; k < n_order; ++k) {
    uint32_t id = UINT32_MAX;
    switch (order[k]) {
      case 0: id = s->scene->add_mesh(s->verts, s->faces); break;
      case 1: id = s->scene->add_spheres(s->sph_c, s->sph_r); break;
      case 2: id = s->scene->add_planes(s->pl_c, s->pl_dx, s->pl_dy, s->pl_rot); break;
      case 3: id = s->scene->add_cylinders(s->cy_c, s->cy_a, s->cy_b, s->cy_h, s->cy_rot); break;
    }
    if (geom_ids) geom_ids[k] = id;
  }
  const auto t0 = std::chrono::steady_clock::now();
  s->scene->commit();
  s->commit_seconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return s;
}

double ref_scene_commit_seconds(void *h) { return static_cast<RefScene *>(h)->commit_seconds; }

void ref_scene_destroy(void *h) { delete static_cast<RefScene *>(h); }

// intersect1 over n rays.  Misses leave the default RayHit (blazert/ray.h:80-84).
// nthreads <= 0 uses the OpenMP default.  Returns wall seconds of the ray loop.
double ref_scene_intersect_ex(void *h, long n, const double *org, const double *dir,
                              const double *tmin, const double *tmax, int any_hit, double *t,
                              double *uv, double *normal, uint32_t *prim, uint32_t *geom,
                              uint8_t *hit, int nthreads);

double ref_scene_intersect(void *h, long n, const double *org, const double *dir,
                           const double *tmin, const double *tmax, double *t, double *uv,
                           double *normal, uint32_t *prim, uint32_t *geom, uint8_t *hit,
                           int nthreads) {
  return ref_scene_intersect_ex(h, n, org, dir, tmin, tmax, 0, t, uv, normal, prim, geom, hit,
                                nthreads);
}

// As ref_scene_intersect, every ray built with Ray::AnyHit::yes when any_hit is non-zero.
double ref_scene_intersect_ex(void *h, long n, const double *org, const double *dir,
                              const double *tmin, const double *tmax, int any_hit, double *t,
                              double *uv, double *normal, uint32_t *prim, uint32_t *geom,
                              uint8_t *hit, int nthreads) {
  const RefScene *s = static_cast<RefScene *>(h);
  const BlazertScene<double> &scene = *s->scene;
  const long row = 512;
  const long rows = (n + row - 1) / row;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  const auto t0 = std::chrono::steady_clock::now();
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (long r = 0; r < rows; ++r) {
    const long end = (r + 1) * row < n ? (r + 1) * row : n;
    for (long i = r * row; i < end; ++i) {
      const Ray<double> ray{v3(org + 3 * i), v3(dir + 3 * i),
                            tmin ? tmin[i] : 0.0,
                            tmax ? tmax[i] : std::numeric_limits<double>::max(),
                            Ray<double>::CullBackFace::no,
                            any_hit ? Ray<double>::AnyHit::yes : Ray<double>::AnyHit::no};
      RayHit<double> rh;
      const bool hh = intersect1(scene, ray, rh);
      if (t) t[i] = rh.hit_distance;
      if (uv) {
        uv[2 * i] = rh.uv[0];
        uv[2 * i + 1] = rh.uv[1];
      }
      if (normal)
        for (int k = 0; k < 3; ++k) normal[3 * i + k] = rh.normal[k];
      if (prim) prim[i] = rh.prim_id;
      if (geom) geom[i] = rh.geom_id;
      if (hit) hit[i] = hh ? 1 : 0;
    }
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Tree dump for node-by-node comparison with the product's builder.  Call once with bmin == NULL
// to get the node count, then with arrays sized for it (prim_ids sized by the primitive count).
long ref_scene_tree(void *h, int kind, double *bmin, double *bmax, uint32_t *leaf, uint32_t *axis,
                    uint32_t *children, uint32_t *prim_off, uint32_t *prim_cnt, uint32_t *prim_ids,
                    long prim_cap) {
  const RefScene *s = static_cast<RefScene *>(h);
  switch (kind) {
    case 0:
      return dump_tree<TriangleMesh>(s, bmin, bmax, leaf, axis, children, prim_off, prim_cnt,
                                     prim_ids, prim_cap);
    case 1:
      return dump_tree<SphereCollection>(s, bmin, bmax, leaf, axis, children, prim_off, prim_cnt,
                                         prim_ids, prim_cap);
    case 2:
      return dump_tree<PlaneCollection>(s, bmin, bmax, leaf, axis, children, prim_off, prim_cnt,
                                        prim_ids, prim_cap);
    case 3:
      return dump_tree<CylinderCollection>(s, bmin, bmax, leaf, axis, children, prim_off,
                                           prim_cnt, prim_ids, prim_cap);
  }
  return -1;
}

// The reference's own per-primitive distance_to_surface (blazert/primitives/sphere.h:179-182,
// plane.h:272-284, cylinder.h:677-759) on primitive ids[i] of one kind for n points.  For
// triangles, whose distance_to_surface (trimesh.h:183-192) cannot be instantiated, the
// reference's closest_point_on_triangle (trimesh_distance.h:177-218) on the face's vertices,
// norm(closest - p) as the distance and the point in closest (n x 3, may be NULL).
void ref_distance_to_surface(void *h, int kind, long n, const uint32_t *ids, const double *points,
                             double *distance, double *closest) {
  const RefScene *s = static_cast<RefScene *>(h);
  for (long i = 0; i < n; ++i) {
    const Vec3r<double> p = v3(points + 3 * i);
    const unsigned id = ids[i];
    switch (kind) {
      case 0: {
        const Vec3ui &f = s->faces[id];
        const Vec3r<double> c =
            closest_point_on_triangle(s->verts[f[0]], s->verts[f[1]], s->verts[f[2]], p);
        distance[i] = norm(c - p);
        if (closest)
          for (int k = 0; k < 3; ++k) closest[3 * i + k] = c[k];
        break;
      }
      case 1:
        distance[i] = distance_to_surface(
            primitive_from_collection(bvh_of<SphereCollection>(s)->collection, id), p);
        break;
      case 2:
        distance[i] = distance_to_surface(
            primitive_from_collection(bvh_of<PlaneCollection>(s)->collection, id), p);
        break;
      case 3:
        distance[i] = distance_to_surface(
            primitive_from_collection(bvh_of<CylinderCollection>(s)->collection, id), p);
        break;
    }
  }
}

// ref_distance_to_surface over n pairs with OpenMP over the pairs: the CPU baseline of the
// distance kernel.  Returns the seconds of the loop.
double ref_distance_to_surface_timed(void *h, int kind, long n, const uint32_t *ids,
                                     const double *points, double *distance, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  const long chunk = 4096;
  const auto t0 = std::chrono::steady_clock::now();
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (long b = 0; b < n; b += chunk) {
    const long m = std::min(chunk, n - b);
    ref_distance_to_surface(h, kind, m, ids + b, points + 3 * b, distance + b, nullptr);
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// The nearest surface of the scene by a loop over every primitive with the reference's own
// distance functions (kinds in the order triangles, spheres, planes, cylinders, ids increasing,
// the first strictly smaller value kept): what a caller of the reference computes without a
// scene-level query.  OpenMP over the points; returns the seconds of the loop.
double ref_closest_surface_timed(void *h, long n, const double *points, double *distance,
                                 uint32_t *prim, uint32_t *geom, int nthreads) {
  const RefScene *s = static_cast<RefScene *>(h);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  const long counts[4] = {long(s->faces.size()), long(s->sph_r.size()), long(s->pl_dx.size()),
                          long(s->cy_a.size())};
  const bool present[4] = {s->scene->has_triangles, s->scene->has_spheres, s->scene->has_planes,
                           s->scene->has_cylinders};
  const uint32_t geom_ids[4] = {present[0] ? s->scene->triangles_geom_id : UINT32_MAX,
                                present[1] ? s->scene->spheres_geom_id : UINT32_MAX,
                                present[2] ? s->scene->planes_geom_id : UINT32_MAX,
                                present[3] ? s->scene->cylinders_geom_id : UINT32_MAX};
  const auto t0 = std::chrono::steady_clock::now();
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16)
#endif
  for (long i = 0; i < n; ++i) {
    double best = std::numeric_limits<double>::infinity();
    uint32_t bp = UINT32_MAX, bg = UINT32_MAX;
    for (int kind = 0; kind < 4; ++kind) {
      if (!present[kind]) continue;
      for (long id = 0; id < counts[kind]; ++id) {
        const uint32_t u = uint32_t(id);
        double d = 0.0;
        ref_distance_to_surface(h, kind, 1, &u, points + 3 * i, &d, nullptr);
        if (d < best) {
          best = d;
          bp = u;
          bg = geom_ids[kind];
        }
      }
    }
    distance[i] = best;
    if (prim) prim[i] = bp;
    if (geom) geom[i] = bg;
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int ref_build_statistics(void *h, int kind, uint32_t *out) {
  const RefScene *s = static_cast<RefScene *>(h);
  switch (kind) {
    case 0: return build_statistics<TriangleMesh>(s, out);
    case 1: return build_statistics<SphereCollection>(s, out);
    case 2: return build_statistics<PlaneCollection>(s, out);
    case 3: return build_statistics<CylinderCollection>(s, out);
  }
  return -1;
}

// Traversal of ONE per-type BVH (blazert/bvh/accel.h:60-120) for n rays, as the reference's
// benchmarks time it (benchmarks/benchmark_BVH/realistic/benchmark_BVH_traverse.cpp:33-60).
double ref_scene_traverse_kind(void *h, int kind, long n, const double *org, const double *dir,
                               double *t, uint32_t *prim, uint8_t *hit, int nthreads) {
  const RefScene *s = static_cast<RefScene *>(h);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  const auto t0 = std::chrono::steady_clock::now();
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 512)
#endif
  for (long i = 0; i < n; ++i) {
    const Ray<double> ray{v3(org + 3 * i), v3(dir + 3 * i)};
    RayHit<double> rh;
    bool hh = false;
    switch (kind) {
      case 0: hh = traverse(*bvh_of<TriangleMesh>(s), ray, rh); break;
      case 1: hh = traverse(*bvh_of<SphereCollection>(s), ray, rh); break;
      case 2: hh = traverse(*bvh_of<PlaneCollection>(s), ray, rh); break;
      case 3: hh = traverse(*bvh_of<CylinderCollection>(s), ray, rh); break;
    }
    t[i] = rh.hit_distance;
    prim[i] = rh.prim_id;
    hit[i] = hh;
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // extern "C"
