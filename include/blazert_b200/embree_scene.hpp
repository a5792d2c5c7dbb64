// EmbreeScene-compatible facade (blazert/embree/scene.h:33-88, :102-140): the same class and
// free intersect1 over blazert_b200's GPU path, so that call sites written for the reference's
// Embree backend compile with a namespace change.
//
// EmbreeScene<double> is the reference's double path exactly: its add_* and intersect1 forward
// to the blazeRT scene (embree/scene.h's double branches call BlazertScene), here
// blazert_b200::Scene<double>, with the same bit-exact results.
// EmbreeScene<float> takes float geometry and rays and answers with the double-precision path
// on the widened inputs, results rounded to float.  Embree itself is not part of this build:
// its float BVH and traversal, its unnormalised geometric normal and its barycentric uv are
// NOT reproduced; hit/miss, prim_id, geom_id and distances are those of the exact
// double-precision query of the same geometry.
#pragma once

#include <type_traits>
#include <vector>

#include "scene.hpp"

namespace blazert_b200 {

template <typename T>
class EmbreeScene {
  static_assert(std::is_same<T, float>::value || std::is_same<T, double>::value,
                "EmbreeScene<float> or EmbreeScene<double>");

 public:
  Scene<double> blazertscene;
  bool has_been_committed = false;

  unsigned int add_mesh(const Vec3rList<T> &vertices, const Vec3iList &triangles) {
    return blazertscene.add_mesh(widen(vertices), triangles);
  }
  unsigned int add_spheres(const Vec3rList<T> &centers, const std::vector<T> &radii) {
    return blazertscene.add_spheres(widen(centers), widen(radii));
  }
  unsigned int add_planes(const Vec3rList<T> &centers, const std::vector<T> &dxs,
                          const std::vector<T> &dys, const Mat3rList<T> &rotations) {
    return blazertscene.add_planes(widen(centers), widen(dxs), widen(dys), widen(rotations));
  }
  unsigned int add_cylinders(const Vec3rList<T> &centers, const std::vector<T> &semi_axes_a,
                             const std::vector<T> &semi_axes_b, const std::vector<T> &heights,
                             const Mat3rList<T> &rotations) {
    return blazertscene.add_cylinders(widen(centers), widen(semi_axes_a), widen(semi_axes_b),
                                      widen(heights), widen(rotations));
  }
  // embree/scene.h:76-87: commits once; later calls return the first result
  bool commit() {
    if (!has_been_committed) has_been_committed = blazertscene.commit();
    return has_been_committed;
  }

 private:
  static const Vec3rList<double> &widen(const Vec3rList<double> &v) { return v; }
  static const std::vector<double> &widen(const std::vector<double> &v) { return v; }
  static const Mat3rList<double> &widen(const Mat3rList<double> &v) { return v; }
  static Vec3rList<double> widen(const Vec3rList<float> &v) {
    Vec3rList<double> r(v.size());
    for (size_t i = 0; i < v.size(); ++i) r[i] = {v[i][0], v[i][1], v[i][2]};
    return r;
  }
  static std::vector<double> widen(const std::vector<float> &v) {
    return std::vector<double>(v.begin(), v.end());
  }
  static Mat3rList<double> widen(const Mat3rList<float> &v) {
    Mat3rList<double> r(v.size());
    for (size_t i = 0; i < v.size(); ++i)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) r[i](a, b) = v[i](a, b);
    return r;
  }
};

// embree/scene.h:102-140
template <typename T>
inline bool intersect1(const EmbreeScene<T> &scene, const Ray<T> &ray, RayHit<T> &rayhit) {
  if constexpr (std::is_same<T, double>::value) {
    return intersect1(scene.blazertscene, ray, rayhit);
  } else {
    Ray<double> r{{ray.origin[0], ray.origin[1], ray.origin[2]},
                  {ray.direction[0], ray.direction[1], ray.direction[2]},
                  static_cast<double>(ray.min_hit_distance),
                  static_cast<double>(ray.max_hit_distance)};
    r.any_hit = ray.any_hit == Ray<T>::AnyHit::yes ? Ray<double>::AnyHit::yes
                                                   : Ray<double>::AnyHit::no;
    RayHit<double> h;
    const bool hit = intersect1(scene.blazertscene, r, h);
    if (hit) {
      rayhit.normal = {float(h.normal[0]), float(h.normal[1]), float(h.normal[2])};
      rayhit.uv = {float(h.uv[0]), float(h.uv[1])};
      rayhit.hit_distance = float(h.hit_distance);
      rayhit.prim_id = h.prim_id;
      rayhit.geom_id = h.geom_id;
    }
    return hit;
  }
}

}  // namespace blazert_b200
