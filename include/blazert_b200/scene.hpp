// blazert_b200 C++ facade: blazeRT's Scene API (blazert/scene.h, blazert/ray.h) over the
// C-ABI of libblazert_b200.so, so that reference-style call sites compile with a namespace
// change.  Header-only; link with -lblazert_b200.
//
// Types mirror the reference's aliases (blazert/datatypes.h:31-59) with standard containers:
// Vec3r<T> = std::array<T, 3>, Vec3rList<T> = std::vector<Vec3r<T>>, Mat3r<T> a row-major 3x3
// with nested-brace construction.  T = double is the reference's double path bit for bit;
// T = float widens to it (see Scene).
#pragma once

#include <array>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <limits>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../blazert_b200.h"

namespace blazert_b200 {

template <typename T>
using Vec3r = std::array<T, 3>;
template <typename T>
using Vec2r = std::array<T, 2>;
using Vec3ui = std::array<unsigned int, 3>;
template <typename T>
using Vec3rList = std::vector<Vec3r<T>>;
using Vec3iList = std::vector<Vec3ui>;

template <typename T>
struct Mat3r {
  T m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  Mat3r() = default;
  Mat3r(std::initializer_list<std::initializer_list<T>> rows) {
    int i = 0;
    for (const auto &row : rows) {
      int j = 0;
      for (const T &x : row) m[i][j++] = x;
      ++i;
    }
  }
  static Mat3r identity() { return Mat3r{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}; }
  T &operator()(size_t i, size_t j) { return m[i][j]; }
  const T &operator()(size_t i, size_t j) const { return m[i][j]; }
};
template <typename T>
using Mat3rList = std::vector<Mat3r<T>>;

// blazert/ray.h:19-65: the direction need not be unit length.  AnyHit::yes ends each kind's
// traversal at its first accepted hit; CullBackFace is accepted and, as in the reference
// (ray.h:52), has no effect.
template <typename T>
struct Ray {
  enum class CullBackFace { yes, no };
  enum class AnyHit { yes, no };
  Vec3r<T> origin;
  Vec3r<T> direction;
  T min_hit_distance = T(0);
  T max_hit_distance = std::numeric_limits<T>::max();
  CullBackFace cull_back_face = CullBackFace::no;
  AnyHit any_hit = AnyHit::no;
  Ray(const Vec3r<T> &o, const Vec3r<T> &d, T tmin = T(0),
      T tmax = std::numeric_limits<T>::max(), CullBackFace cull = CullBackFace::no,
      AnyHit any = AnyHit::no)
      : origin(o), direction(d), min_hit_distance(tmin), max_hit_distance(tmax),
        cull_back_face(cull), any_hit(any) {}
};

// blazert/ray.h:72-85, with the reference's defaults.
template <typename T>
struct RayHit {
  Vec3r<T> normal{0, 0, 0};
  Vec2r<T> uv{0, 0};
  T hit_distance = std::numeric_limits<T>::max();
  unsigned int prim_id = static_cast<unsigned int>(-1);
  unsigned int geom_id = static_cast<unsigned int>(-1);
};

// blazert/ray.h:86-120: the same field dump.  The reference's Ray keeps the normalised
// direction, its inverse and signs from its constructor (ray.h:56-65); this Ray keeps the raw
// direction, so they are formed here the same way for the dump.
template <typename T>
std::ostream &operator<<(std::ostream &stream, const Ray<T> &ray) {
  const T len = std::sqrt((ray.direction[0] * ray.direction[0] +
                           ray.direction[1] * ray.direction[1]) +
                          ray.direction[2] * ray.direction[2]);
  const T inv_len = T(1) / len;
  stream << "{\n";
  stream << "  Ray: " << &ray << ",\n";
  stream << "  origin: [" << ray.origin[0] << "," << ray.origin[1] << "," << ray.origin[2]
         << "],\n";
  stream << "  direction: [" << ray.direction[0] * inv_len << "," << ray.direction[1] * inv_len
         << "," << ray.direction[2] * inv_len << "],\n";
  stream << "  direction_inv: [" << T(1) / ray.direction[0] << "," << T(1) / ray.direction[1]
         << "," << T(1) / ray.direction[2] << "],\n";
  stream << "  direction_sign: [" << (ray.direction[0] < T(0)) << "," << (ray.direction[1] < T(0))
         << "," << (ray.direction[2] < T(0)) << "],\n";
  stream << "  min_hit_distance: " << ray.min_hit_distance << ",\n";
  stream << "  max_hit_distance " << ray.max_hit_distance << ",\n";
  stream << "  cull_back_face "
         << (ray.cull_back_face == Ray<T>::CullBackFace::no ? "no" : "yes") << ",\n";
  stream << "  any_hit: " << (ray.any_hit == Ray<T>::AnyHit::no ? "no" : "yes") << "\n";
  stream << "}\n";
  return stream;
}

// blazert/ray.h:105-118
template <typename T>
std::ostream &operator<<(std::ostream &stream, const RayHit<T> &rayhit) {
  stream << "{\n";
  stream << "  Ray: " << &rayhit << ",\n";
  stream << "  normal: [" << rayhit.normal[0] << "," << rayhit.normal[1] << ","
         << rayhit.normal[2] << "],\n";
  stream << "  uv: [" << rayhit.uv[0] << "," << rayhit.uv[1] << "],\n";
  stream << "  hit_distance: " << rayhit.hit_distance << ",\n";
  stream << "  prim_id: " << rayhit.prim_id << ",\n";
  stream << "  geom_id: " << rayhit.geom_id << ",\n";
  stream << "}\n";
  return stream;
}

// blazert/bvh/options.h:15-29
template <typename T>
struct BVHBuildOptions {
  unsigned int min_leaf_primitives = 4;
  unsigned int max_tree_depth = 28;
  unsigned int bin_size = 64;
};

// blazert/bvh/statistics.h:11-38, member for member (the reference's builder returns it;
// Scene::build_statistics gives it per kind after commit).
template <typename T>
struct BVHBuildStatistics {
  unsigned int max_tree_depth = 0;
  unsigned int leaf_nodes = 0;
  unsigned int max_num_prims_per_leaf = 0;
  unsigned int min_num_prims_per_leaf = static_cast<unsigned int>(-1);
  unsigned int branch_nodes = 0;
  unsigned int bad_splits = 0;
  std::chrono::duration<T> build_time{T(0)};
};

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string &what) : std::runtime_error(what), code(code) {}
  int code;
};

inline void check(int rc) {
  if (rc != BZR_OK) throw Error(rc, bzr_last_error_string());
}

// blazert/scene.h:38-115.  Scene<double> is the reference's double path, bit for bit.
// Scene<float> accepts the reference's float call sites and answers with the double-precision
// query of the widened geometry and rays, rounded to float (not the reference's float BVH and
// traversal, which this build does not reproduce).
template <typename T>
class Scene {
  static_assert(std::is_same<T, double>::value || std::is_same<T, float>::value,
                "Scene<double> or Scene<float>");

 public:
  BVHBuildOptions<T> build_options;

  Scene() { check(bzr_scene_create(&s_)); }
  ~Scene() { bzr_scene_destroy(s_); }
  Scene(const Scene &) = delete;
  Scene &operator=(const Scene &) = delete;

  // Each returns the geom id, or static_cast<unsigned>(-1) for a second add of a kind or an
  // add after commit (as the reference does); other errors throw blazert_b200::Error.
  unsigned int add_mesh(const Vec3rList<T> &vertices_in, const Vec3iList &triangles) {
    const auto &vertices = wide(vertices_in);
    uint32_t id = 0;
    const int rc = bzr_add_mesh(s_, flat(vertices), vertices.size(),
                                reinterpret_cast<const uint32_t *>(triangles.data()),
                                triangles.size(), &id);
    return added(rc, id);
  }
  unsigned int add_spheres(const Vec3rList<T> &centers_in, const std::vector<T> &radii_in) {
    const auto &centers = wide(centers_in);
    const auto &radii = wide(radii_in);
    uint32_t id = 0;
    if (centers.size() != radii.size()) throw Error(BZR_EINVAL, "centers and radii differ");
    const int rc = bzr_add_spheres(s_, flat(centers), radii.data(), radii.size(), &id);
    return added(rc, id);
  }
  unsigned int add_planes(const Vec3rList<T> &centers_in, const std::vector<T> &dxs_in,
                          const std::vector<T> &dys_in, const Mat3rList<T> &rotations_in) {
    const auto &centers = wide(centers_in);
    const auto &dxs = wide(dxs_in);
    const auto &dys = wide(dys_in);
    const auto &rotations = wide(rotations_in);
    uint32_t id = 0;
    const size_t n = centers.size();
    if (dxs.size() != n || dys.size() != n || rotations.size() != n)
      throw Error(BZR_EINVAL, "plane arrays differ in length");
    const int rc =
        bzr_add_planes(s_, flat(centers), dxs.data(), dys.data(), flat(rotations), n, &id);
    return added(rc, id);
  }
  unsigned int add_cylinders(const Vec3rList<T> &centers_in, const std::vector<T> &a_in,
                             const std::vector<T> &b_in, const std::vector<T> &heights_in,
                             const Mat3rList<T> &rotations_in) {
    const auto &centers = wide(centers_in);
    const auto &semi_axes_a = wide(a_in);
    const auto &semi_axes_b = wide(b_in);
    const auto &heights = wide(heights_in);
    const auto &rotations = wide(rotations_in);
    uint32_t id = 0;
    const size_t n = centers.size();
    if (semi_axes_a.size() != n || semi_axes_b.size() != n || heights.size() != n ||
        rotations.size() != n)
      throw Error(BZR_EINVAL, "cylinder arrays differ in length");
    const int rc = bzr_add_cylinders(s_, flat(centers), semi_axes_a.data(), semi_axes_b.data(),
                                     heights.data(), flat(rotations), n, &id);
    return added(rc, id);
  }

  bool commit() {
    const bzr_build_options o{build_options.min_leaf_primitives, build_options.max_tree_depth,
                              build_options.bin_size};
    check(bzr_commit(s_, &o));
    return true;
  }

  // Batched query, structure of arrays of doubles (see bzr_intersectN_ex); returns nothing,
  // fills outputs.  ray_flags: 0 or BZR_RAY_ANY_HIT for every ray.
  void intersectN(size_t n, const double *origins, const double *directions,
                  const double *tmin, const double *tmax, double *hit_distance, double *uv,
                  double *normal, uint32_t *prim_id, uint32_t *geom_id, uint8_t *hit,
                  int mode = BZR_MODE_FP64, void *stream = nullptr,
                  uint32_t ray_flags = 0) const {
    check(bzr_intersectN_ex(s_, n, origins, directions, tmin, tmax, hit_distance, uv, normal,
                            prim_id, geom_id, hit, mode, ray_flags, stream));
  }

  // Distances (bzr_distance_to_surface): kind 0 triangles, 1 spheres, 2 planes, 3 cylinders;
  // closest (triangles only) may be null.
  void distance_to_surface(int kind, size_t n, const uint32_t *prim_ids, const double *points,
                           double *distance, double *closest = nullptr,
                           void *stream = nullptr) const {
    check(bzr_distance_to_surface(s_, kind, n, prim_ids, points, distance, closest, stream));
  }
  // Nearest surface of the scene per point (bzr_closest_surface).
  void closest_surface(size_t n, const double *points, double *distance, uint32_t *prim_id,
                       uint32_t *geom_id, void *stream = nullptr) const {
    check(bzr_closest_surface(s_, n, points, distance, prim_id, geom_id, stream));
  }

  // Persistent format (bzr_scene_save / bzr_scene_load): a loaded scene is committed and
  // answers as the saved one, without rebuilding its trees.
  void save(const std::string &path) const { check(bzr_scene_save(s_, path.c_str())); }
  static std::unique_ptr<Scene> load(const std::string &path) {
    bzr_scene *h = nullptr;
    check(bzr_scene_load(&h, path.c_str()));
    return std::unique_ptr<Scene>(new Scene(h));
  }

  // Build statistics of one kind's BVH (0 triangles, 1 spheres, 2 planes, 3 cylinders).
  BVHBuildStatistics<T> build_statistics(int kind) const {
    bzr_build_statistics b;
    check(bzr_scene_build_statistics(s_, kind, &b));
    BVHBuildStatistics<T> st;
    st.max_tree_depth = b.max_tree_depth;
    st.leaf_nodes = b.leaf_nodes;
    st.max_num_prims_per_leaf = b.max_num_prims_per_leaf;
    st.min_num_prims_per_leaf = b.min_num_prims_per_leaf;
    st.branch_nodes = b.branch_nodes;
    st.bad_splits = b.bad_splits;
    st.build_time = std::chrono::duration<T>(static_cast<T>(b.build_seconds));
    return st;
  }

  const bzr_scene *handle() const { return s_; }

 private:
  explicit Scene(bzr_scene *h) : s_(h) {}
  template <typename V>
  static const double *flat(const std::vector<V> &v) {
    static_assert(sizeof(V) % sizeof(double) == 0, "contiguous double storage");
    return reinterpret_cast<const double *>(v.data());
  }
  // double inputs pass through; float inputs are widened
  static const Vec3rList<double> &wide(const Vec3rList<double> &v) { return v; }
  static const std::vector<double> &wide(const std::vector<double> &v) { return v; }
  static const Mat3rList<double> &wide(const Mat3rList<double> &v) { return v; }
  static Vec3rList<double> wide(const Vec3rList<float> &v) {
    Vec3rList<double> r(v.size());
    for (size_t i = 0; i < v.size(); ++i) r[i] = {v[i][0], v[i][1], v[i][2]};
    return r;
  }
  static std::vector<double> wide(const std::vector<float> &v) {
    return std::vector<double>(v.begin(), v.end());
  }
  static Mat3rList<double> wide(const Mat3rList<float> &v) {
    Mat3rList<double> r(v.size());
    for (size_t i = 0; i < v.size(); ++i)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) r[i](a, b) = v[i](a, b);
    return r;
  }
  static unsigned int added(int rc, uint32_t id) {
    if (rc == BZR_ESTATE) return static_cast<unsigned int>(-1);
    check(rc);
    return id;
  }
  bzr_scene *s_ = nullptr;
};

// blazert/scene.h:161-210.  Starts from a default RayHit: the reference compares later kinds
// against the caller's incoming rayhit.hit_distance (scene.h:181), which equals the default
// for the fresh RayHit every reference example and test passes.
template <typename T>
inline bool intersect1(const Scene<T> &scene, const Ray<T> &ray, RayHit<T> &rayhit) {
  bzr_rayhit rh;
  int hit = 0;
  const uint32_t flags = ray.any_hit == Ray<T>::AnyHit::yes ? BZR_RAY_ANY_HIT : 0u;
  const double o[3] = {ray.origin[0], ray.origin[1], ray.origin[2]};
  const double d[3] = {ray.direction[0], ray.direction[1], ray.direction[2]};
  check(bzr_intersect1_ex(scene.handle(), o, d, ray.min_hit_distance, ray.max_hit_distance,
                          flags, &rh, &hit));
  if (hit) {
    rayhit.normal = {T(rh.normal[0]), T(rh.normal[1]), T(rh.normal[2])};
    rayhit.uv = {T(rh.uv[0]), T(rh.uv[1])};
    rayhit.hit_distance = T(rh.hit_distance);
    rayhit.prim_id = rh.prim_id;
    rayhit.geom_id = rh.geom_id;
  }
  return hit != 0;
}

}  // namespace blazert_b200
