// Known-answer capture for the reference's own test files (test infrastructure, oracle only).
//
// oracle/Makefile force-includes this header (-include) into each reference test file it
// compiles.  It includes the reference headers and the reference's assert helpers
// (test/test_primitives/assert_helper.h) first and then declares explicit specialisations of
// those helpers for T = double.  Each specialisation
//   * records the collection, the ray (or query point) and the values the test asserts
//     (expected hit, prim id, distance, normal, box, centre, distance to surface) as one JSON
//     line, and
//   * evaluates the reference exactly as the helper does -- prepare_traversal +
//     intersect_primitive + post_traversal on primitive 0, or SAHBinnedBuilder + traverse --
//     and records those outputs too, then runs the helper's CHECKs.
// The node-test cases of test/test_bvh/test_intersect.cpp are captured by a specialisation of
// intersect_node that forwards to the reference's own template (through a node type of ours).
// The float instantiations are not captured (the GPU path is double precision).
#pragma once
#include <blazert/bvh/accel.h>
#include <blazert/bvh/builder.h>
#include <blazert/bvh/intersect.h>
#include <blazert/datatypes.h>
#include <blazert/primitives/cylinder.h>
#include <blazert/primitives/plane.h>
#include <blazert/primitives/sphere.h>
#include <blazert/primitives/trimesh.h>
#include <blazert/ray.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "assert_helper.h"

namespace kat {

inline std::FILE *&sink() {
  static std::FILE *f = nullptr;
  return f;
}

inline std::string num(double x) {
  if (std::isnan(x)) return "NaN";
  if (std::isinf(x)) return x > 0 ? "Infinity" : "-Infinity";
  if (x == 0.0) return std::signbit(x) ? "-0.0" : "0.0";  // keep the sign of zero through JSON
  char b[40];
  std::snprintf(b, sizeof b, "%.17g", x);
  return b;
}
inline std::string str(const std::string &s) {
  std::string o = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') o += '\\';
    o += c;
  }
  return o + "\"";
}
template <class V>
inline std::string vec(const V &v, int n) {
  std::string o = "[";
  for (int i = 0; i < n; ++i) o += (i ? "," : "") + num(double(v[i]));
  return o + "]";
}
inline std::string vlist(const blazert::Vec3rList<double> &l) {
  std::string o = "[";
  for (size_t i = 0; i < l.size(); ++i) o += (i ? "," : "") + vec(l[i], 3);
  return o + "]";
}
inline std::string slist(const std::vector<double> &l) {
  std::string o = "[";
  for (size_t i = 0; i < l.size(); ++i) o += (i ? "," : "") + num(l[i]);
  return o + "]";
}
inline std::string mlist(const blazert::Mat3rList<double> &l) {
  std::string o = "[";
  for (size_t i = 0; i < l.size(); ++i) {
    o += i ? "," : "";
    o += "[";
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) o += ((r || c) ? "," : "") + num(l[i](r, c));
    o += "]";
  }
  return o + "]";
}

inline std::string geometry(const blazert::TriangleMesh<double> &m) {
  std::string f = "[";
  for (size_t i = 0; i < m.faces.size(); ++i)
    f += (i ? ",[" : "[") + std::to_string(m.faces[i][0]) + "," + std::to_string(m.faces[i][1]) +
         "," + std::to_string(m.faces[i][2]) + "]";
  return "\"kind\":\"mesh\",\"vertices\":" + vlist(m.vertices) + ",\"faces\":" + f + "]";
}
inline std::string geometry(const blazert::SphereCollection<double> &s) {
  return "\"kind\":\"spheres\",\"centers\":" + vlist(s.centers) + ",\"radii\":" + slist(s.radii);
}
inline std::string geometry(const blazert::PlaneCollection<double> &p) {
  return "\"kind\":\"planes\",\"centers\":" + vlist(p.centers) + ",\"dxs\":" + slist(p.dxs) +
         ",\"dys\":" + slist(p.dys) + ",\"rotations\":" + mlist(p.rotations);
}
inline std::string geometry(const blazert::CylinderCollection<double> &c) {
  return "\"kind\":\"cylinders\",\"centers\":" + vlist(c.centers) + ",\"semi_axes_a\":" +
         slist(c.semi_axes_a) + ",\"semi_axes_b\":" + slist(c.semi_axes_b) + ",\"heights\":" +
         slist(c.heights) + ",\"rotations\":" + mlist(c.rotations);
}

// The raw direction the test passed is not stored by Ray (blazert/ray.h:52-62).  It is
// recovered from 1 / direction_inv: per component the doubles within a few ulps whose inverse
// is exactly direction_inv, and of those combinations the one whose normalisation is exactly
// the stored direction.  "direction_exact" says whether such a raw direction was found.
inline std::string ray(const blazert::Ray<double> &r) {
  std::vector<double> cand[3];
  for (int i = 0; i < 3; ++i) {
    const double first = 1.0 / r.direction_inv[i];
    cand[i].push_back(first);  // exact for zeros (1 / +-inf) and most test values
    double x = first;
    for (int k = 0; k < 4; ++k) x = std::nextafter(x, -std::numeric_limits<double>::infinity());
    for (int k = 0; k < 9; ++k, x = std::nextafter(x, std::numeric_limits<double>::infinity())) {
      const double inv = 1.0 / x;
      if (x != first && std::isfinite(inv) && !std::memcmp(&inv, &r.direction_inv[i], 8))
        cand[i].push_back(x);
    }
  }
  blazert::Vec3r<double> raw{cand[0][0], cand[1][0], cand[2][0]};
  bool exact = false;
  for (double a : cand[0])
    for (double b : cand[1])
      for (double c : cand[2]) {
        if (exact) break;
        const blazert::Vec3r<double> t{a, b, c};
        const blazert::Vec3r<double> n = normalize(t);
        bool same = true;
        for (int i = 0; i < 3; ++i) {
          const double inv = 1.0 / t[i];
          if (std::memcmp(&inv, &r.direction_inv[i], 8) || std::memcmp(&n[i], &r.direction[i], 8))
            same = false;
        }
        if (same) {
          raw = t;
          exact = true;
        }
      }
  return "\"origin\":" + vec(r.origin, 3) + ",\"direction\":" + vec(raw, 3) +
         ",\"direction_exact\":" + (exact ? "true" : "false") +
         ",\"tmin\":" + num(r.min_hit_distance) + ",\"tmax\":" + num(r.max_hit_distance);
}

inline std::string hit(bool h, const blazert::RayHit<double> &rh) {
  return "{\"hit\":" + std::string(h ? "true" : "false") + ",\"prim_id\":" +
         std::to_string(rh.prim_id) + ",\"distance\":" + num(rh.hit_distance) +
         ",\"normal\":" + vec(rh.normal, 3) + ",\"uv\":" + vec(rh.uv, 2) + "}";
}

inline void emit(const std::string &what, const std::string &body) {
  if (!sink()) return;
  std::fprintf(sink(), "{\"case\":%s,\"check\":%s,%s}\n",
               str(doctest::detail::subcase_path()).c_str(), str(what).c_str(), body.c_str());
}

template <template <typename> class Coll>
void primitive_hit(const Coll<double> &collection, const blazert::Ray<double> &r, bool true_hit,
                   unsigned prim_id, double distance, const blazert::Vec3r<double> &normal,
                   bool check_prim) {
  typename Coll<double>::intersector intersector(collection);
  blazert::RayHit<double> rayhit;
  prepare_traversal(intersector, r);
  const bool h = intersect_primitive(intersector, primitive_from_collection(collection, 0), r);
  if (h) post_traversal(intersector, rayhit);
  emit("intersect_primitive",
       geometry(collection) + "," + kat::ray(r) + ",\"expected\":{\"hit\":" +
           (true_hit ? "true" : "false") + ",\"prim_id\":" + std::to_string(prim_id) +
           ",\"distance\":" + num(distance) + ",\"normal\":" + vec(normal, 3) +
           ",\"check_prim\":" + (check_prim ? "true" : "false") + "},\"reference\":" + hit(h, rayhit));
  CHECK(h == true_hit);
  if (check_prim) CHECK(rayhit.prim_id == prim_id);
  CHECK(rayhit.hit_distance == doctest::Approx(distance));
  CHECK(rayhit.normal[0] == doctest::Approx(normal[0]));
  CHECK(rayhit.normal[1] == doctest::Approx(normal[1]));
  CHECK(rayhit.normal[2] == doctest::Approx(normal[2]));
}

// mode: 0 full (prim id + normal), 1 no prim id, 2 distance only, 3 hit only (a WARN)
template <template <typename> class Coll>
void traverse_hit(const Coll<double> &collection, const blazert::Ray<double> &r, bool true_hit,
                  unsigned prim_id, double distance, const blazert::Vec3r<double> &normal,
                  int mode) {
  blazert::BVH<double, Coll> bvh(collection);
  blazert::SAHBinnedBuilder builder;
  builder.build(bvh);
  blazert::RayHit<double> rayhit;
  const bool h = traverse(bvh, r, rayhit);
  emit("traverse",
       geometry(collection) + "," + kat::ray(r) + ",\"expected\":{\"hit\":" +
           (true_hit ? "true" : "false") + ",\"prim_id\":" + std::to_string(prim_id) +
           ",\"distance\":" + num(distance) + ",\"normal\":" + vec(normal, 3) +
           ",\"mode\":" + std::to_string(mode) + "},\"reference\":" + hit(h, rayhit));
  if (mode == 3) {
    WARN(h == true_hit);
    return;
  }
  CHECK(h == true_hit);
  if (mode == 0) CHECK(rayhit.prim_id == prim_id);
  CHECK(rayhit.hit_distance == doctest::Approx(distance));
  if (mode <= 1) {
    CHECK(rayhit.normal[0] == doctest::Approx(normal[0]));
    CHECK(rayhit.normal[1] == doctest::Approx(normal[1]));
    CHECK(rayhit.normal[2] == doctest::Approx(normal[2]));
  }
}

template <template <typename> class Coll>
void box(const Coll<double> &collection, unsigned prim_id, const blazert::Vec3r<double> &mn,
         const blazert::Vec3r<double> &mx) {
  const auto [bmin, bmax] = collection.get_primitive_bounding_box(prim_id);
  emit("bounding_box", geometry(collection) + ",\"prim_id\":" + std::to_string(prim_id) +
                           ",\"expected\":{\"min\":" + vec(mn, 3) + ",\"max\":" + vec(mx, 3) +
                           "},\"reference\":{\"min\":" + vec(bmin, 3) + ",\"max\":" + vec(bmax, 3) + "}");
  for (int k = 0; k < 3; ++k) {
    CHECK(bmin[k] == doctest::Approx(mn[k]));
    CHECK(bmax[k] == doctest::Approx(mx[k]));
  }
}

template <template <typename> class Coll>
void center(const Coll<double> &collection, unsigned prim_id, const blazert::Vec3r<double> &c) {
  const auto got = collection.get_primitive_center(prim_id);
  emit("center", geometry(collection) + ",\"prim_id\":" + std::to_string(prim_id) +
                     ",\"expected\":" + vec(c, 3) + ",\"reference\":" + vec(got, 3));
  for (int k = 0; k < 3; ++k) CHECK(got[k] == doctest::Approx(c[k]));
}

struct Node {
  blazert::Vec3r<double> min, max;
};

// assert_distance_to_surface (test/test_primitives/assert_helper.h:102-106): the reference's
// distance_to_surface of one primitive and the test's expected value.
template <template <typename> class Coll>
void distance(const Coll<double> &collection, unsigned prim_id, const blazert::Vec3r<double> &p,
              double true_distance) {
  const double got = distance_to_surface(primitive_from_collection(collection, prim_id), p);
  emit("distance_to_surface", geometry(collection) + ",\"prim_id\":" + std::to_string(prim_id) +
                                  ",\"point\":" + vec(p, 3) + ",\"expected\":" +
                                  num(true_distance) + ",\"reference\":" + num(got));
  CHECK(got == doctest::Approx(true_distance));
}

}  // namespace kat

#define KAT_SPECIALISE(COLL)                                                                      \
  template <>                                                                                     \
  inline void assert_intersect_primitive_hit<double, blazert::COLL>(                              \
      const blazert::COLL<double> &c, const blazert::Ray<double> &r, const bool h,               \
      const unsigned int p, const double d, const blazert::Vec3r<double> &n) {                    \
    kat::primitive_hit<blazert::COLL>(c, r, h, p, d, n, true);                                    \
  }                                                                                               \
  template <>                                                                                     \
  inline void assert_traverse_bvh_hit<double, blazert::COLL>(                                     \
      const blazert::COLL<double> &c, const blazert::Ray<double> &r, const bool h,               \
      const unsigned int p, const double d, const blazert::Vec3r<double> &n) {                    \
    kat::traverse_hit<blazert::COLL>(c, r, h, p, d, n, 0);                                        \
  }                                                                                               \
  template <>                                                                                     \
  inline void assert_traverse_bvh_hit_collection<double, blazert::COLL>(                          \
      const blazert::COLL<double> &c, const blazert::Ray<double> &r, const bool h,               \
      const double d, const blazert::Vec3r<double> &n) {                                          \
    kat::traverse_hit<blazert::COLL>(c, r, h, 0, d, n, 1);                                        \
  }                                                                                               \
  template <>                                                                                     \
  inline void assert_traverse_bvh_hit_trimesh_distance<double, blazert::COLL>(                    \
      const blazert::COLL<double> &c, const blazert::Ray<double> &r, const bool h,               \
      const double d) {                                                                           \
    kat::traverse_hit<blazert::COLL>(c, r, h, 0, d, blazert::Vec3r<double>{0., 0., 0.}, 2);       \
  }                                                                                               \
  template <>                                                                                     \
  inline void assert_traverse_bvh_hit_trimesh_precision<double, blazert::COLL>(                   \
      const blazert::COLL<double> &c, const blazert::Ray<double> &r, const bool h,               \
      const double, const double) {                                                               \
    kat::traverse_hit<blazert::COLL>(c, r, h, 0, 0.0, blazert::Vec3r<double>{0., 0., 0.}, 3);     \
  }                                                                                               \
  template <>                                                                                     \
  inline void assert_bounding_box<double, blazert::COLL>(                                         \
      const blazert::COLL<double> &c, const unsigned int p, const blazert::Vec3r<double> &mn,    \
      const blazert::Vec3r<double> &mx) {                                                         \
    kat::box<blazert::COLL>(c, p, mn, mx);                                                        \
  }                                                                                               \
  template <>                                                                                     \
  inline void assert_primitive_center<double, blazert::COLL>(                                     \
      const blazert::COLL<double> &c, const unsigned int p, const blazert::Vec3r<double> &ctr) { \
    kat::center<blazert::COLL>(c, p, ctr);                                                        \
  }

KAT_SPECIALISE(TriangleMesh)
KAT_SPECIALISE(SphereCollection)
KAT_SPECIALISE(PlaneCollection)
KAT_SPECIALISE(CylinderCollection)
#undef KAT_SPECIALISE

// The reference's tests assert distances for spheres, planes and cylinders (its triangle
// distance_to_surface cannot be instantiated, and no test calls it).
#define KAT_SPECIALISE_DISTANCE(COLL)                                                             \
  template <>                                                                                     \
  inline void assert_distance_to_surface<double, blazert::COLL>(                                  \
      const blazert::COLL<double> &c, const unsigned int p, const blazert::Vec3r<double> &pt,   \
      const double d) {                                                                           \
    kat::distance<blazert::COLL>(c, p, pt, d);                                                    \
  }
KAT_SPECIALISE_DISTANCE(SphereCollection)
KAT_SPECIALISE_DISTANCE(PlaneCollection)
KAT_SPECIALISE_DISTANCE(CylinderCollection)
#undef KAT_SPECIALISE_DISTANCE

// test/test_bvh/test_intersect.cpp tests intersect_node on BVHNode<T, PlaneCollection>.
template <>
inline bool blazert::intersect_node<double, blazert::BVHNode<double, blazert::PlaneCollection>>(
    double &min_distance, double &max_distance,
    const blazert::BVHNode<double, blazert::PlaneCollection> &node,
    const blazert::Ray<double> &ray) noexcept {
  const kat::Node n{node.min, node.max};
  const double in_min = min_distance, in_max = max_distance;
  const bool h = blazert::intersect_node<double, kat::Node>(min_distance, max_distance, n, ray);
  if (doctest::detail::state().test_case == "Intersect_node")
    kat::emit("intersect_node", "\"bmin\":" + kat::vec(node.min, 3) + ",\"bmax\":" +
                                    kat::vec(node.max, 3) + "," + kat::ray(ray) +
                                    ",\"in\":[" + kat::num(in_min) + "," + kat::num(in_max) +
                                    "],\"reference\":{\"hit\":" + (h ? "true" : "false") +
                                    ",\"tmin\":" + kat::num(min_distance) + ",\"tmax\":" +
                                    kat::num(max_distance) + "}");
  return h;
}
