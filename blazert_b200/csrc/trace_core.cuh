// Per-ray closest-hit traversal, shared by the sm_100a kernels (trace.cu) and, compiled as
// host code, by the test-only CPU emulator (tests/emu/).  Exactness rules are stated in
// trace.cu.  Everything here is a pure function of the scene view and one ray.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>

#include "layout.h"

#if defined(__CUDACC__)
#include <cuda_runtime.h>
#include <math_constants.h>
#define BZR_HD __host__ __device__ __forceinline__
#define BZR_INF (__builtin_inf())
#else
#include <vector_types.h>
#include <vector_functions.h>
using std::isfinite;
using std::isnan;
#define BZR_HD inline
#define BZR_INF (__builtin_inf())
#endif

namespace bzr {

// Portability shims: the same source runs as device code and as host code.
template <class T>
BZR_HD T ldg(const T *p) {
#if defined(__CUDA_ARCH__)
  return __ldg(p);
#else
  return *p;
#endif
}
BZR_HD void flag_error(uint32_t *err, uint32_t bit) {
#if defined(__CUDA_ARCH__)
  atomicOr(err, bit);
#else
  *err |= bit;
#endif
}
BZR_HD long long dbits(double x) {
#if defined(__CUDA_ARCH__)
  return __double_as_longlong(x);
#else
  long long r;
  std::memcpy(&r, &x, 8);
  return r;
#endif
}
BZR_HD double bitsd(long long x) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double(x);
#else
  double r;
  std::memcpy(&r, &x, 8);
  return r;
#endif
}

constexpr double kL1 = 1.0 + 4.0 * 2.220446049250313080847e-16;  // 1 + 4 * DBL_EPSILON
constexpr double kTol = 4.0 * 2.220446049250313080847e-16;      // trimesh.h:156
constexpr double kDblMax = 1.7976931348623157e308;

struct D3 {
  double x, y, z;
};
BZR_HD D3 d3(double a, double b, double c) { return {a, b, c}; }
BZR_HD D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
BZR_HD D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
BZR_HD D3 mul(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
BZR_HD D3 divs(D3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
BZR_HD double dot(D3 a, D3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
BZR_HD D3 cross(D3 a, D3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
BZR_HD double norm(D3 a) { return sqrt(dot(a, a)); }
BZR_HD D3 normalize(D3 a) {
  const double len = norm(a);
  return mul(a, len != 0.0 ? 1.0 / len : 0.0);
}
// R * v and trans(R) * v for a row-major 3x3 R
BZR_HD D3 rot(const double *R, D3 v) {
  return {(R[0] * v.x + R[1] * v.y) + R[2] * v.z, (R[3] * v.x + R[4] * v.y) + R[5] * v.z,
          (R[6] * v.x + R[7] * v.y) + R[8] * v.z};
}
BZR_HD D3 rot_t(const double *R, D3 v) {
  return {(R[0] * v.x + R[3] * v.y) + R[6] * v.z, (R[1] * v.x + R[4] * v.y) + R[7] * v.z,
          (R[2] * v.x + R[5] * v.y) + R[8] * v.z};
}
// x with its sign flipped when y is negative (blazert/datatypes.h:83-85)
BZR_HD double product_sign(double x, double y) {
  return bitsd(dbits(x) ^ (dbits(y) & (long long)0x8000000000000000ULL));
}

struct Ray {
  D3 o, d, inv;  // origin, normalized direction, 1 / raw direction
  unsigned sx, sy, sz;
  double tmin, tmax;
  bool any_hit;  // Ray::AnyHit::yes (blazert/ray.h:24-34)
};

// blazert/ray.h:56-65
BZR_HD Ray make_ray(const double *o, const double *raw, double tmin,
                                        double tmax) {
  Ray r;
  r.o = d3(o[0], o[1], o[2]);
  const D3 w = d3(raw[0], raw[1], raw[2]);
  r.d = normalize(w);
  r.inv = d3(1.0 / w.x, 1.0 / w.y, 1.0 / w.z);
  r.sx = w.x < 0.0;
  r.sy = w.y < 0.0;
  r.sz = w.z < 0.0;
  r.tmin = tmin;
  r.tmax = tmax;
  r.any_hit = false;
  return r;
}

// One axis of the slab test; lo/hi are the box's bounds on that axis.
BZR_HD void slab_axis(double lo, double hi, unsigned s, double o, double inv,
                                          double &mn, double &mx, bool &nan) {
  const double entry = s ? hi : lo;
  const double exit = s ? lo : hi;
  const double a = (entry - o) * inv;
  const double b = ((exit - o) * inv) * kL1;
  mn = (a < mn) ? mn : a;  // std::max(a, mn)
  nan |= (b != b);
  mx = (mx < b) ? mx : b;  // std::min(b, mx)
}

// Hit-independent part of intersect_node for a box given as (lo, hi) pairs per axis.
// Returns whether the box can be accepted for some hit distance; *key is the entry distance
// to compare with the hit distance at pop time (-inf when the reference ignores it).
BZR_HD bool box_test(double2 px, double2 py, double2 pz, const Ray &r,
                                         double &key) {
  double mn = r.tmin, mx = BZR_INF;
  bool nan = false;
  slab_axis(px.x, px.y, r.sx, r.o.x, r.inv.x, mn, mx, nan);
  slab_axis(py.x, py.y, r.sy, r.o.y, r.inv.y, mn, mx, nan);
  slab_axis(pz.x, pz.y, r.sz, r.o.z, r.inv.z, mn, mx, nan);
  key = nan ? -BZR_INF : mn;
  return mn <= mx;
}

// Per-kind intersector state (the reference's *Intersector after prepare_traversal).
struct KState {
  double hit;     // intersector.hit_distance
  double u, v;    // uv (triangles only; 0 otherwise)
  uint32_t pos;   // leaf-order position of the primitive hit
  D3 n;           // plane / cylinder normal as computed at hit time (not yet normalized)
};

BZR_HD double2 ld2(const double *p) {
  return ldg(reinterpret_cast<const double2 *>(p));
}

// 32 bytes at p (32-byte aligned) as two uint4, kept in L2 with priority on the device.
BZR_HD void ld32_keep(const void *p, uint4 &a, uint4 &b) {
#if defined(__CUDA_ARCH__)
  asm("ld.global.nc.L2::evict_last.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
      : "l"(p));
#else
  std::memcpy(&a, p, 16);
  std::memcpy(&b, static_cast<const char *>(p) + 16, 16);
#endif
}

// One 32-byte load of a 32-byte aligned {x, y, z, w} entry (vertices, vertex normals).
BZR_HD D3 ld_d4xyz(const double *p) {
#if defined(__CUDA_ARCH__)
  double x, y, z, w;
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(x), "=d"(y), "=d"(z), "=d"(w) : "l"(p));
  (void)w;
  return d3(x, y, z);
#else
  return d3(p[0], p[1], p[2]);
#endif
}

BZR_HD D3 ld_vertex(const double *verts, uint32_t i) {
  return ld_d4xyz(verts + size_t(i) * kVertexDoubles);
}

// blazert/primitives/trimesh.h:153-181, the quantities of one test before its decisions.  F
// holds the triangle's three vertex indices; v0, e1 = v0 - v1, e2 = v2 - v0 (the reference
// Triangle's members, trimesh.h:19-31) and n = cross(e1, e2) are formed here with the
// reference's operations, hence the same bits.
struct TriTest {
  double u, v, w, det, abs_det;  // unnormalised barycentrics, det and |det|
  D3 n, c;                       // for the unnormalised distance product_sign(dot(n, c), det)
};
BZR_HD TriTest tri_test(const double *verts, uint4 F, const Ray &r) {
  const D3 v0 = ld_vertex(verts, F.x), v1 = ld_vertex(verts, F.y), v2 = ld_vertex(verts, F.z);
  const D3 e1 = sub(v0, v1), e2 = sub(v2, v0);
  TriTest q;
  q.n = cross(e1, e2);
  q.c = sub(v0, r.o);
  const D3 rr = cross(r.d, q.c);
  q.det = dot(q.n, r.d);
  q.abs_det = fabs(q.det);
  q.u = product_sign(dot(rr, e2), q.det);
  q.v = product_sign(dot(rr, e1), q.det);
  q.w = (q.abs_det - q.u) - q.v;
  return q;
}

// The whole test.  UV: store the hit's barycentrics in st (the mixed-precision walk leaves
// them out while it walks and forms them once at the end, tri_uv).
template <bool UV = true>
BZR_HD bool isect_triangle(const double *verts, uint4 F, uint32_t pos, const Ray &r,
                           KState &st) {
  const TriTest q = tri_test(verts, F, r);
  if (q.u >= -kTol && q.v >= -kTol && q.w >= -kTol) {
    const double t = product_sign(dot(q.n, q.c), q.det);
    if (t >= q.abs_det * r.tmin && q.abs_det * st.hit > t) {
      const double inv_det = 1.0 / q.abs_det;
      st.hit = t * inv_det;
      if (UV) {
        st.u = q.u * inv_det;
        st.v = q.v * inv_det;
      }
      st.pos = pos;
      return true;
    }
  }
  return false;
}

// The barycentrics isect_triangle<true> stores for the triangle at leaf position st.pos (the
// same operations, hence the same bits).
BZR_HD void tri_uv(const KindView &K, const Ray &r, KState &st) {
  const TriTest q = tri_test(K.verts, ldg(reinterpret_cast<const uint4 *>(K.tri) + st.pos), r);
  const double inv_det = 1.0 / q.abs_det;
  st.u = q.u * inv_det;
  st.v = q.v * inv_det;
}

// blazert/primitives/sphere.h:135-177
BZR_HD bool isect_sphere(const double *P, uint32_t pos, const Ray &r,
                                             KState &st) {
  const double2 q0 = ld2(P), q1 = ld2(P + 2);
  const D3 center = d3(q0.x, q0.y, q1.x);
  const double radius = q1.y;
  const D3 v = sub(r.o, center);
  const double A = dot(r.d, r.d);
  const double B = 2.0 * dot(v, r.d);
  const double C = dot(v, v) - radius * radius;
  const double D = B * B - (4.0 * A) * C;
  if (D < 0.0) return false;
  const double Q = sqrt(D);
  const double rcpA = 1.0 / A;
  const double t0 = (0.5 * rcpA) * (-B - Q);
  const double t1 = (0.5 * rcpA) * (-B + Q);
  if ((t0 > r.tmin) && (t0 < st.hit)) {
    st.hit = norm(mul(r.d, t0));
    st.pos = pos;
    return true;
  }
  if ((t1 > r.tmin) && (t1 < st.hit)) {
    st.hit = norm(mul(r.d, t1));
    st.pos = pos;
    return true;
  }
  return false;
}

// blazert/primitives/plane.h:180-270
BZR_HD bool isect_plane(const double *P, uint32_t pos, const Ray &r,
                                            KState &st) {
  double R[9];
  const double2 q0 = ld2(P), q1 = ld2(P + 2), q2 = ld2(P + 4), q3 = ld2(P + 6), q4 = ld2(P + 8),
                q5 = ld2(P + 10), q6 = ld2(P + 12);
  const D3 center = d3(q0.x, q0.y, q1.x);
  const double dx = q1.y, dy = q2.x;
  R[0] = q2.y; R[1] = q3.x; R[2] = q3.y; R[3] = q4.x; R[4] = q4.y;
  R[5] = q5.x; R[6] = q5.y; R[7] = q6.x; R[8] = q6.y;
  const D3 org = rot_t(R, sub(r.o, center));
  const D3 dir = rot_t(R, r.d);
  const double t1 = -org.z / dir.z;
  if (!((t1 > r.tmin) && (t1 < st.hit))) return false;
  const D3 ic = add(org, mul(dir, t1));
  const double x_min = -dx / 2, x_max = dx / 2, y_min = -dy / 2, y_max = dy / 2;
  const double x = ic.x, y = ic.y;
  const double sz = org.z / fabs(org.z);
  D3 n;
  if ((x > x_min) && (x < x_max) && (y > y_min) && (y < y_max)) {
    const D3 ez = rot(R, d3(0.0, 0.0, 1.0));
    n = d3(sz * ez.x, sz * ez.y, sz * ez.z);
  } else if ((x == x_min) && (x < x_max) && (y > y_min) && (y < y_max)) {  // edges
    n = rot(R, d3(-1.0, 0.0, sz));
  } else if ((x > x_min) && (x == x_max) && (y > y_min) && (y < y_max)) {
    n = rot(R, d3(1.0, 0.0, sz));
  } else if ((x > x_min) && (x < x_max) && (y == y_min) && (y < y_max)) {
    n = rot(R, d3(0.0, -1.0, sz));
  } else if ((x > x_min) && (x < x_max) && (y > y_min) && (y == y_max)) {
    n = rot(R, d3(0.0, 1.0, sz));
  } else if ((x == x_min) && (x < x_max) && (y == y_min) && (y < y_max)) {  // corners
    n = rot(R, d3(-1.0, -1.0, sz));
  } else if ((x == x_min) && (x < x_max) && (y > y_min) && (y == y_max)) {
    n = rot(R, d3(-1.0, 1.0, sz));
  } else if ((x > x_min) && (x == x_max) && (y == y_min) && (y < y_max)) {
    n = rot(R, d3(1.0, -1.0, sz));
  } else if ((x > x_min) && (x == x_max) && (y > y_min) && (y == y_max)) {
    n = rot(R, d3(1.0, 1.0, sz));
  } else {
    return false;
  }
  st.n = n;
  st.hit = norm(mul(dir, t1));
  st.pos = pos;
  return true;
}

// Result of one cylinder test: the reference's post-hit state (the normal as computed at hit
// time and norm(t * dir) as the hit distance).
struct CylHit {
  bool hit;
  double dist;
  D3 n;
};

BZR_HD CylHit cyl_hit(D3 n, double t, D3 dir) { return CylHit{true, norm(mul(dir, t)), n}; }
BZR_HD CylHit cyl_miss() { return CylHit{false, 0.0, d3(0.0, 0.0, 0.0)}; }

// blazert/primitives/cylinder.h:181-495 (no hit-distance test; unrotated normal in one branch).
// Takes the ray's origin and direction and returns its result by value, so that nothing of the
// caller's ray or state has to live in memory around the test.
BZR_HD CylHit isect_cylinder(const double *P, D3 ro, D3 rd) {
  double R[9];
  const double2 q0 = ld2(P), q1 = ld2(P + 2), q2 = ld2(P + 4), q3 = ld2(P + 6), q4 = ld2(P + 8),
                q5 = ld2(P + 10), q6 = ld2(P + 12), q7 = ld2(P + 14);
  const D3 center = d3(q0.x, q0.y, q1.x);
  const double a = q1.y, b = q2.x, h = q2.y;
  R[0] = q3.x; R[1] = q3.y; R[2] = q4.x; R[3] = q4.y; R[4] = q5.x;
  R[5] = q5.y; R[6] = q6.x; R[7] = q6.y; R[8] = q7.x;
  const D3 org = rot_t(R, sub(ro, center));
  const D3 dir = rot_t(R, rd);
  const double x0 = org.x, y0 = org.y, z0 = org.z;
  const double j = dir.x, k = dir.y, l = dir.z;
  const double h2 = h / 2.0, mh2 = -h / 2.0;
  auto ng = [&](D3 n) { return divs(rot(R, n), norm(n)); };
  auto shell_n = [&](D3 ic) { return d3(2 * ic.x / (a * a), 2 * ic.y / (b * b), 0.0); };
  // the elliptic-shell quadratic, in the reference's operation order
  auto quad = [&](double &t0, double &t1, D3 &i0, D3 &i1) {
    const double A = a * a * k * k + b * b * j * j;
    const double B = a * a * k * y0 + b * b * j * x0;
    const double C = a * a * k * k + b * b * j * j - j * j * y0 * y0 + 2 * j * k * x0 * y0 -
                     k * k * x0 * x0;
    if (C < 0) return false;
    const double rA = 1.0 / A;  // -1.0 / A is -(1.0 / A) exactly
    const double s = a * b * sqrt(C);
    t0 = rA * (-B + s);
    t1 = -rA * (B + s);
    i0 = add(org, mul(dir, t0));
    i1 = add(org, mul(dir, t1));
    return true;
  };
  double t0, t1;
  D3 i0, i1;
  if (z0 > h2 || z0 < mh2) {  // areas 1 and 2: origin above or below the caps
    if (l == 0) return cyl_miss();
    const double zc = z0 > h2 ? h2 : mh2;
    const double tc = (zc - z0) / l;
    if (tc < 0) return cyl_miss();
    const D3 ic = add(org, mul(dir, tc));
    if (b * b * ic.x * ic.x + a * a * ic.y * ic.y <= a * a * b * b)
      return cyl_hit(ng(d3(0.0, 0.0, z0 > h2 ? 1.0 : -1.0)), tc, dir);
    if (!quad(t0, t1, i0, i1)) return cyl_miss();
    if ((t1 > 0) && (t1 < t0) && (i1.z <= h2) && (i1.z >= mh2))
      return cyl_hit(ng(shell_n(i1)), t1, dir);
    if ((t0 > 0) && (t0 < t1) && (i0.z <= h2) && (i0.z >= mh2))
      return cyl_hit(ng(shell_n(i0)), t0, dir);
    return cyl_miss();  // area 4 cannot hold when z0 is outside [-h/2, h/2]
  }
  const double ell = x0 * x0 * b * b + y0 * y0 * a * a;
  if ((z0 > mh2) && (z0 < h2) && (ell > a * a * b * b)) {  // area 3: beside the shell
    if (!quad(t0, t1, i0, i1)) return cyl_miss();
    if ((t1 > 0) && (t1 < t0) && (i1.z <= h2) && (i1.z >= mh2))
      return cyl_hit(ng(shell_n(i1)), t1, dir);
    if ((t0 > 0) && (t0 < t1) && (i0.z <= h2) && (i0.z >= mh2))
      return cyl_hit(ng(shell_n(i0)), t0, dir);
    return cyl_miss();
  }
  if ((z0 >= mh2) && (z0 <= h2) && (ell <= a * a * b * b)) {  // area 4: inside
    if (l == 0) {
      if ((z0 == mh2) || (z0 == h2)) return cyl_miss();
      if (!quad(t0, t1, i0, i1)) return cyl_miss();
      if ((t1 > 0) && (i1.z <= h2) && (i1.z >= mh2))
        return cyl_hit(ng(shell_n(i1)), t1, dir);
      if ((t0 > 0) && (i0.z <= h2) && (i0.z >= mh2))
        return cyl_hit(ng(shell_n(i0)), t0, dir);
    } else if ((j == 0.0) && (k == 0)) {
      if (b * b * x0 * x0 + a * a * y0 * y0 == a * a * b * b) return cyl_miss();
      if (l < 0) return cyl_hit(ng(d3(0.0, 0.0, -1.0)), (mh2 - z0) / l, dir);
      if (l > 0) return cyl_hit(ng(d3(0.0, 0.0, 1.0)), (h2 - z0) / l, dir);
    } else {
      if (!quad(t0, t1, i0, i1)) return cyl_miss();
      if ((t1 > 0) && (i1.z <= h2) && (i1.z >= mh2))
        return cyl_hit(ng(shell_n(i1)), t1, dir);
      if ((t0 > 0) && (i0.z <= h2) && (i0.z >= mh2))
        return cyl_hit(shell_n(i0), t0, dir);  // unrotated (cylinder.h:462-463)
      if (l < 0) return cyl_hit(ng(d3(0.0, 0.0, -1.0)), (mh2 - z0) / l, dir);
      if (l > 0) return cyl_hit(ng(d3(0.0, 0.0, 1.0)), (h2 - z0) / l, dir);
    }
  }
  return cyl_miss();
}

// Tests the primitive at leaf position pos and returns its id word (id | kLastBit on the
// leaf's last primitive); hit receives intersect_primitive's result.
template <int KIND>
BZR_HD uint32_t isect(const KindView &K, uint32_t pos, const Ray &r, KState &st, bool &hit) {
  if (KIND == kMesh) {
    const uint4 F = ldg(reinterpret_cast<const uint4 *>(K.tri) + pos);
    hit = isect_triangle(K.verts, F, pos, r, st);
    return F.w;
  }
  const uint32_t id = ldg(K.prim_ids + pos);
  const double *P = K.payload + size_t(pos) * kPayloadDoubles[KIND];
  if (KIND == kSpheres) {
    hit = isect_sphere(P, pos, r, st);
  } else if (KIND == kPlanes) {
    hit = isect_plane(P, pos, r, st);
  } else {
    const CylHit c = isect_cylinder(P, r.o, r.d);
    hit = c.hit;
    if (c.hit) {  // no closest-hit test (blazert/primitives/cylinder.h:181-495)
      st.n = c.n;
      st.hit = c.dist;
      st.pos = pos;
    }
  }
  return id;
}

// Traversal storage of a thread: the stack (entry j of thread t at [j * stride + t]; stride 1
// for a thread-local array), and the first n_top nodes of the walked node array (FP64 nodes,
// or wide nodes on the mixed path; the top levels, as nodes are numbered breadth-first)
// staged in shared memory by the block, 8 x 16 bytes each.
struct Stack {
  double *key;
  uint32_t *ref;
  uint32_t cap, stride;
  const uint4 *top = nullptr;
  uint32_t n_top = 0;
};

BZR_HD double2 as_d2(uint4 q) {
  double2 d;
  std::memcpy(&d, &q, sizeof d);
  return d;
}

// Work counters of one ray (counting kernels only), per kind: box tests (FP64 path: the
// reference's node pops, i.e. the root plus both children of every accepted internal node;
// mixed path: the root plus every child slot tested), primitive tests, node fetches (internal
// FP64 nodes, or wide nodes) and leaf fetches (FP64 path: leaves whose primitives run; mixed
// path: leaf records read, each with its exact FP64 test).
struct Counts {
  uint32_t box[kNumKinds];
  uint32_t prim[kNumKinds];
  uint32_t node[kNumKinds];
  uint32_t leaf[kNumKinds];
};

// Resumable traversal of one kind (blazert/bvh/accel.h:80-120).  trav_begin tests the root;
// trav_to_leaf walks internal nodes until the current reference is a leaf; trav_leaf runs the
// leaf's primitives (blazert/bvh/intersect.h:67-78) and pops the next accepted entry.  The
// persistent kernels interleave these steps across the lanes of a warp; traverse() runs them
// to completion.
struct Trav {
  uint32_t cur;  // node index, or kLeafBit | first primitive position of a leaf
  uint32_t sp;   // stack depth
  bool live;     // false once the stack is exhausted
  // wide walk only: the leaf records found and not yet processed, in visit order (kNoLeaf:
  // none; post2 is set only after post), and whether cur still holds a reference to walk
  uint32_t post, post2;
  bool walk;
};
constexpr uint32_t kNoLeaf = 0xFFFFFFFFu;  // no leaf record has this reference

// Whether `pred` holds for some lane of the warp among `lanes` (device); for the single ray of
// a host call, pred itself.
BZR_HD bool warp_any(unsigned lanes, bool pred) {
#if defined(__CUDA_ARCH__)
  return __any_sync(lanes, pred);
#else
  (void)lanes;
  return pred;
#endif
}
BZR_HD unsigned active_lanes() {
#if defined(__CUDA_ARCH__)
  return __activemask();
#else
  return 1u;
#endif
}

template <int KIND, bool COUNT>
BZR_HD void trav_begin(const KindView &K, const Ray &r, KState &st, Trav &tv, Counts *cnt) {
  st.hit = r.tmax;  // prepare_traversal
  st.u = st.v = 0.0;
  st.pos = 0xFFFFFFFFu;
  st.n = d3(0.0, 0.0, 0.0);
  tv.sp = 0;
  tv.cur = K.root_ref;
  double key;
  const double2 bx = make_double2(K.root_box[0], K.root_box[1]);
  const double2 by = make_double2(K.root_box[2], K.root_box[3]);
  const double2 bz = make_double2(K.root_box[4], K.root_box[5]);
  if (COUNT) cnt->box[KIND] += 1;
  tv.live = box_test(bx, by, bz, r, key) && !(key > st.hit);
}

// Pops until an entry passes its deferred hit-distance test; ends the traversal otherwise.
BZR_HD void trav_pop(Trav &tv, const KState &st, const Stack &sk, uint32_t tid) {
  while (tv.sp > 0) {
    --tv.sp;
    if (!(sk.key[tv.sp * sk.stride + tid] > st.hit)) {
      tv.cur = sk.ref[tv.sp * sk.stride + tid];
      return;
    }
  }
  tv.live = false;
}

template <int KIND, bool COUNT>
BZR_HD void trav_to_leaf(const KindView &K, const Ray &r, const KState &st, Trav &tv,
                         const Stack &sk, uint32_t tid, uint32_t *err, Counts *cnt) {
  while (tv.live && !(tv.cur & kLeafBit)) {
    if (tv.cur >= K.n_internal) {
      flag_error(err, kErrNodeIndex);
      tv.live = false;
      return;
    }
    double2 a0, a1, a2, b0, b1, b2;
    uint4 meta;
    if (tv.cur < sk.n_top) {  // a top-level node staged in shared memory
      const uint4 *q = sk.top + size_t(tv.cur) * 8;
      a0 = as_d2(q[0]), a1 = as_d2(q[1]), a2 = as_d2(q[2]);
      b0 = as_d2(q[3]), b1 = as_d2(q[4]), b2 = as_d2(q[5]);
      meta = q[6];
    } else {
      const double *nd = K.nodes64 + size_t(tv.cur) * kNode64Doubles;
      uint4 w0, w1, w2, w3, w4, w5;  // the two child boxes in three 32-byte loads
      ld32_keep(nd, w0, w1);
      ld32_keep(nd + 4, w2, w3);
      ld32_keep(nd + 8, w4, w5);
      a0 = as_d2(w0), a1 = as_d2(w1), a2 = as_d2(w2);
      b0 = as_d2(w3), b1 = as_d2(w4), b2 = as_d2(w5);
      meta = ldg(reinterpret_cast<const uint4 *>(nd + 12));
    }
    double k0, k1;
    if (COUNT) {
      cnt->box[KIND] += 2;
      cnt->node[KIND] += 1;
    }
    const bool p0 = box_test(a0, a1, a2, r, k0);
    const bool p1 = box_test(b0, b1, b2, r, k1);
    const unsigned near = meta.z == 0 ? r.sx : (meta.z == 1 ? r.sy : r.sz);
    const bool pn = near ? p1 : p0, pf = near ? p0 : p1;
    const double kn = near ? k1 : k0, kf = near ? k0 : k1;
    const uint32_t rn = near ? meta.y : meta.x, rf = near ? meta.x : meta.y;
    if (pf) {  // far child pushed first, as the reference does
      if (tv.sp >= sk.cap) {
        flag_error(err, kErrStack);
        tv.live = false;
        return;
      }
      sk.key[tv.sp * sk.stride + tid] = kf;
      sk.ref[tv.sp * sk.stride + tid] = rf;
      ++tv.sp;
    }
    if (pn && !(kn > st.hit)) {  // the near child is popped next, with the same hit distance
      tv.cur = rn;
    } else {
      trav_pop(tv, st, sk, tid);
    }
  }
}

template <int KIND, bool COUNT>
BZR_HD void trav_leaf(const KindView &K, const Ray &r, KState &st, Trav &tv, const Stack &sk,
                      uint32_t tid, uint32_t *err, Counts *cnt) {
  uint32_t pos = tv.cur & kIdMask;
  if (COUNT) cnt->leaf[KIND] += 1;
  for (;;) {
    if (pos >= K.n_prims) {
      flag_error(err, kErrPrimIndex);
      tv.live = false;
      return;
    }
    if (COUNT) cnt->prim[KIND] += 1;
    bool h;
    const uint32_t id = isect<KIND>(K, pos, r, st, h);
    if (h && r.any_hit) {  // the first hit ends the leaf and the traversal (intersect.h:73-75,
      tv.live = false;     // accel.h:109-110)
      return;
    }
    if (id & kLastBit) break;
    ++pos;
  }
  trav_pop(tv, st, sk, tid);
}

// The whole traversal of one kind.  Returns the reference's hit flag.
template <int KIND, bool COUNT>
BZR_HD bool traverse(const KindView &K, const Ray &r, KState &st, const Stack &sk,
                     uint32_t tid, uint32_t *err, Counts *cnt) {
  Trav tv;
  trav_begin<KIND, COUNT>(K, r, st, tv, cnt);
  while (tv.live) {
    trav_to_leaf<KIND, COUNT>(K, r, st, tv, sk, tid, err, cnt);
    if (tv.live) trav_leaf<KIND, COUNT>(K, r, st, tv, sk, tid, err, cnt);
  }
  return st.hit < r.tmax;
}

// ---------------------------------------------------------------------------------------------
// Mixed precision (BZR_MODE_MIXED) for triangles, spheres and planes: the wide image (layout.h,
// kWideBytes).
//
// Internal levels are walked on the wide nodes with FP32 slab tests of the children's
// quantised boxes, which contain their exact boxes.  Every FP32 near-plane distance is
// computed as a lower bound, and every far-plane distance as an upper bound, of the
// reference's FP64 slab distances for the exact box (the error bound E below is subtracted or
// added in the same fused multiply-add).  A child is kept when its FP32 entry distance is at
// most both its FP32 exit distance and the current hit distance rounded up, so every child the
// FP64 traversal accepts is kept.  The kept children are visited in the reference's order (the
// node's permutation for the ray's octant).  A leaf is processed when the reference's exact
// FP64 test of the leaf's own box against the current hit distance passes
// (blazert/bvh/intersect.h:33-51).
//
// Why the results are the FP64 path's: the walk reaches every node the FP64 traversal accepts,
// in the same relative order (the wide tree is the binary tree with treelets contracted, and a
// treelet's children are visited in the binary order).  The FP64 traversal processes a leaf
// iff the leaf's own test passes at its pop time AND every ancestor passed its test at its own
// pop time.  An ancestor's box contains the leaf's box, the rounded slab distances are
// monotone in the box bounds, and the hit distance only decreases for triangles, spheres and
// planes (cylinders, which may move it outward, keep the FP64 traversal); so when a leaf's own
// test passes, no ancestor failed.  The same leaves are therefore processed in the same order
// with the same hit distance, and every primitive test and result is identical.
//
// Error bound, per node and axis: with A = 2^e inv_f, D = (origin - o_hi) - o_lo (the origin
// held as two floats, so it is exact to 2^-48 relative), B = D inv_f and C = B - 2^23 A, the
// distance of a stored bound origin + q 2^e is t = fma(2^23 + q, A, C +- E): the byte q is
// placed in the mantissa of 2^23 with one byte permute, and the fma cancels the 2^23 A parts
// exactly.  Against the real distance T of that bound for the FP64 inverse direction: inv_f,
// the two differences, B and the fma round by at most 5 * 2^-24 * (255 |A| + |B|) in all; C
// and C +- E are of magnitude 2^23 |A| and round by at most |A| / 2 each; the FP64 reference
// rounds T by 2^-49 relative (its l1 factor included).  E = (1 + 2^-10) |A| + 2^-20 |B| +
// 1e-37 covers all of these (and denormal results), so the near distance is below and the far
// distance above the reference's: one grid cell of slack on top of the outward quantisation.
// The bound follows the ray's own magnitudes on each axis: an axis whose direction component
// is tiny has large distances and a large E, but those distances rarely decide the entry or
// the exit.  Rays with a zero, non-finite or large (> 2^40) inverse direction component, an
// origin component beyond 1e18, or a non-finite or huge tmin or a NaN tmax, take the FP64
// traversal.  Then every FP32 value of the test is finite: node coordinates are within 1e18
// (the builder's limit), so 2^e <= 2^54, |A| <= 2^94, 2^23 |A| <= 2^117, |B| <= 2^101, and
// every distance and difference stays below 2^121.
struct RayW {
  float o_hi[3], o_lo[3], inv[3];
  float tmin;    // tmin rounded down
  uint32_t oct;  // sx | sy << 1 | sz << 2
  bool ok;
};

BZR_HD float f32_up(double x) {  // x rounded toward +inf
#if defined(__CUDA_ARCH__)
  return __double2float_ru(x);
#else
  float f = static_cast<float>(x);
  if (static_cast<double>(f) < x) f = nextafterf(f, __builtin_inff());
  return f;
#endif
}
BZR_HD float fbits(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  std::memcpy(&f, &u, 4);
  return f;
#endif
}
BZR_HD float fma32(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  return __fmaf_rn(a, b, c);
#else
  return fmaf(a, b, c);
#endif
}
BZR_HD float f32_down(double x) {  // x rounded toward -inf
#if defined(__CUDA_ARCH__)
  return __double2float_rd(x);
#else
  float f = static_cast<float>(x);
  if (static_cast<double>(f) > x) f = nextafterf(f, -__builtin_inff());
  return f;
#endif
}

BZR_HD RayW make_ray_w(const Ray &r) {
  RayW f;
  const double inv[3] = {r.inv.x, r.inv.y, r.inv.z}, o[3] = {r.o.x, r.o.y, r.o.z};
  bool ok = fabs(r.tmin) <= 1e18 && !isnan(r.tmax);
  for (int a = 0; a < 3; ++a) {
    const double ai = fabs(inv[a]), oa = fabs(o[a]);
    ok = ok && ai > 0.0 && ai <= 0x1p40 && oa <= 1e18;  // false for NaN and infinities
    f.o_hi[a] = static_cast<float>(o[a]);
    f.o_lo[a] = static_cast<float>(o[a] - static_cast<double>(f.o_hi[a]));
    f.inv[a] = static_cast<float>(inv[a]);
  }
  f.tmin = f32_down(r.tmin);
  f.oct = r.sx | (r.sy << 1) | (r.sz << 2);
  f.ok = ok;
  return f;
}

// Next stack entry of the wide walk (entries carry no distance).
BZR_HD void wtrav_pop(Trav &tv, const Stack &sk, uint32_t tid) {
  if (tv.sp > 0) {
    --tv.sp;
    tv.cur = sk.ref[tv.sp * sk.stride + tid];
  } else {
    tv.walk = false;
  }
}

// FP32 bound of the hit distance for the child tests: rounded up, and +0 for a zero distance,
// so that the sign test of the node walk (exit - entry) never meets -0 as an exit distance.
BZR_HD float hit_bound(double h) {
  const float f = f32_up(h);
  return f == 0.0f ? 0.0f : f;
}

// The exact root test (trav_begin), then the walk starts at the wide root.  hl is the hit
// distance rounded up.
template <int KIND, bool COUNT>
BZR_HD void wtrav_begin(const KindView &K, const Ray &r, const RayW &f, KState &st, float &hl,
                        Trav &tv, Counts *cnt) {
  (void)f;
  trav_begin<KIND, COUNT>(K, r, st, tv, cnt);
  tv.cur = K.wide_root_ref;
  tv.post = tv.post2 = kNoLeaf;
  tv.walk = tv.live;
  hl = hit_bound(st.hit);
}

// prmt.b32 in its default mode: byte i of the result is byte (s_i & 7) of the eight bytes
// {b, a} (a's bytes 0-3, b's bytes 4-7), or, when s_i & 8, the sign bit of that byte
// replicated over the byte, where s_i is nibble i of s.
BZR_HD uint32_t prmt(uint32_t a, uint32_t b, uint32_t s) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(s));
  return r;
#else
  const uint64_t src = uint64_t(a) | (uint64_t(b) << 32);
  uint32_t r = 0;
  for (int i = 0; i < 4; ++i) {
    const uint32_t n = (s >> (4 * i)) & 0xFu;
    uint32_t byte = uint32_t(src >> (8 * (n & 7u))) & 0xFFu;
    if (n & 8u) byte = (byte & 0x80u) ? 0xFFu : 0u;
    r |= byte << (8 * i);
  }
  return r;
#endif
}

// 2^23 + byte `b` (0..3, a compile-time constant in the unrolled loops) of `w`, as a float
// (exact: the byte lands in the low mantissa bits of 2^23).
BZR_HD float qbyte(uint32_t w, int b) { return fbits(prmt(w, 0x4B000000u, unsigned(b) | 0x7440u)); }

BZR_HD float max3f(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
#else
  return fmaxf(fmaxf(a, b), c);
#endif
}
BZR_HD float min3f(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
#else
  return fminf(fminf(a, b), c);
#endif
}
// Two independent single-precision fused multiply-adds, each rounded to nearest.
BZR_HD float2 fma2(float2 a, float2 b, float2 c) {
#if defined(__CUDA_ARCH__)
  return __ffma2_rn(a, b, c);
#else
  return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#endif
}
BZR_HD int ffs64(uint64_t x) {  // 1 + index of the lowest set bit; 0 for x == 0
#if defined(__CUDA_ARCH__)
  return __ffsll(static_cast<long long>(x));
#else
  return __builtin_ffsll(static_cast<long long>(x));
#endif
}
BZR_HD int msb64(uint64_t x) {  // index of the highest set bit of x != 0
#if defined(__CUDA_ARCH__)
  return 63 - __clzll(static_cast<long long>(x));
#else
  return 63 - __builtin_clzll(x);
#endif
}
BZR_HD uint32_t fword(float x) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(x);
#else
  uint32_t u;
  std::memcpy(&u, &x, 4);
  return u;
#endif
}

BZR_HD uint32_t pick8(uint4 a, uint4 b, uint32_t slot) {
  const uint4 q = (slot & 4u) ? b : a;
  const uint32_t lo = (slot & 1u) ? q.y : q.x, hi = (slot & 1u) ? q.w : q.z;
  return (slot & 2u) ? hi : lo;
}

// A lane at a leaf reference with room in its queue of two postponed leaves appends the leaf
// and pops the next entry.
BZR_HD void wtrav_postpone(Trav &tv, const Stack &sk, uint32_t tid) {
  if (tv.walk && (tv.cur & kLeafBit) && tv.post2 == kNoLeaf) {
    if (tv.post == kNoLeaf)
      tv.post = tv.cur;
    else
      tv.post2 = tv.cur;
    wtrav_pop(tv, sk, tid);
  }
}

// The wide walk.
//
// Per node, each child slot's near and far distances per axis come from one paired FMA
// (near and far biases side by side); the child is kept when exit - entry has its sign bit
// clear, i.e. when entry <= exit, with the entry raised to tmin and the exit lowered to the hit
// distance (exact as a sign test: every value is finite and the exit is never -0).  The eight
// sign bytes are gathered into two words in slot order and permuted into the ray's visit order
// (the node's permutation for the ray's octant) with two byte permutes; a slot past the last
// child reads as rejected.  The first kept child in visit order becomes current and the other
// kept ones are pushed from the last in order down, so the next in order ends on top of the
// stack, as in the reference's stack.  Stack entries carry no distance: a popped wide node's
// children are tested against the hit distance of that moment, and a popped leaf gets its
// exact test.
//
// Postponed leaves (Aila and Laine, "Understanding the efficiency of ray traversal on GPUs",
// 2009): a lane that reaches a leaf record keeps it (tv.post, then tv.post2) and walks on while
// some lane of the warp has not found one yet, so that the warp's lanes reach their leaf steps
// together; it stops at a third leaf, and its leaf step processes every leaf it holds.  (A
// queue of two measured 8-10 % faster than one on the workloads here; three or four, slower.)
// The walk past a postponed leaf uses the hit distance from before that leaf, which keeps more
// children, never fewer; leaves are still processed in the visit order, each with its exact
// test.  The counting kernels do not walk ahead, so their counts are the walk's own work.
//
// wtrav_node tests one wide node (the lane is at a node: tv.walk and tv.cur not a leaf).
template <int KIND, bool COUNT>
BZR_HD void wtrav_node(const KindView &K, const RayW &f, float hl, Trav &tv, const Stack &sk,
                       uint32_t tid, uint32_t *err, Counts *cnt) {
  const bool sx = f.oct & 1u, sy = f.oct & 2u, sz = f.oct & 4u;
  if (tv.cur >= K.n_wide) {
    flag_error(err, kErrNodeIndex);
    tv.walk = false;
    return;
  }
  const bool staged = tv.cur < sk.n_top;  // a top-level node staged in shared memory
  const uint4 *nd = staged ? sk.top + size_t(tv.cur) * 8
                           : reinterpret_cast<const uint4 *>(K.wide + size_t(tv.cur) * kWideBytes);
  const uint32_t *words = reinterpret_cast<const uint32_t *>(nd);
  uint4 hd, qx, qy, qz, ra, rb;
  uint32_t perm;
  if (staged) {
    hd = nd[0], qx = nd[1], qy = nd[2], qz = nd[3];
    ra = nd[4], rb = nd[5];
    perm = words[24 + f.oct];
  } else {
    ld32_keep(nd, hd, qx);
    ld32_keep(nd + 2, qy, qz);
    ld32_keep(nd + 4, ra, rb);
    perm = ldg(words + 24 + f.oct);
  }
  // per axis t(q) = fma(2^23 + q, A, B - 2^23 A -+ E): a lower bound of the reference's
  // near-plane distance, an upper bound of its far-plane distance
  const float ax = fbits((hd.w & 0xFFu) << 23) * f.inv[0];
  const float ay = fbits((hd.w & 0xFF00u) << 15) * f.inv[1];
  const float az = fbits((hd.w & 0xFF0000u) << 7) * f.inv[2];
  const float bx = ((fbits(hd.x) - f.o_hi[0]) - f.o_lo[0]) * f.inv[0];
  const float by = ((fbits(hd.y) - f.o_hi[1]) - f.o_lo[1]) * f.inv[1];
  const float bz = ((fbits(hd.z) - f.o_hi[2]) - f.o_lo[2]) * f.inv[2];
  const float cx = fma32(-8388608.0f, ax, bx), cy = fma32(-8388608.0f, ay, by);
  const float cz = fma32(-8388608.0f, az, bz);
  constexpr float kRel = 9.5367431640625e-07f, kCell = 1.0009765625f;  // 2^-20, 1 + 2^-10
  const float ex = fma32(kCell, fabsf(ax), kRel * fabsf(bx)) + 1e-37f;
  const float ey = fma32(kCell, fabsf(ay), kRel * fabsf(by)) + 1e-37f;
  const float ez = fma32(kCell, fabsf(az), kRel * fabsf(bz)) + 1e-37f;
  const float2 Ax = make_float2(ax, ax), Ay = make_float2(ay, ay), Az = make_float2(az, az);
  const float2 Bx = make_float2(cx - ex, cx + ex), By = make_float2(cy - ey, cy + ey);
  const float2 Bz = make_float2(cz - ez, cz + ez);
  // near and far bound words per axis: the hi bounds are near for a negative direction
  const uint32_t nx0 = sx ? qx.z : qx.x, nx1 = sx ? qx.w : qx.y;
  const uint32_t fx0 = sx ? qx.x : qx.z, fx1 = sx ? qx.y : qx.w;
  const uint32_t ny0 = sy ? qy.z : qy.x, ny1 = sy ? qy.w : qy.y;
  const uint32_t fy0 = sy ? qy.x : qy.z, fy1 = sy ? qy.y : qy.w;
  const uint32_t nz0 = sz ? qz.z : qz.x, nz1 = sz ? qz.w : qz.y;
  const uint32_t fz0 = sz ? qz.x : qz.z, fz1 = sz ? qz.y : qz.w;
  uint32_t sgn[8];  // exit - entry per slot (its sign bit: rejected)
#pragma unroll
  for (int c = 0; c < kWideMax; ++c) {
    const int b = c & 3;
    const float2 tx = fma2(make_float2(qbyte(c < 4 ? nx0 : nx1, b), qbyte(c < 4 ? fx0 : fx1, b)),
                           Ax, Bx);
    const float2 ty = fma2(make_float2(qbyte(c < 4 ? ny0 : ny1, b), qbyte(c < 4 ? fy0 : fy1, b)),
                           Ay, By);
    const float2 tz = fma2(make_float2(qbyte(c < 4 ? nz0 : nz1, b), qbyte(c < 4 ? fz0 : fz1, b)),
                           Az, Bz);
    const float entry = max3f(tx.x, ty.x, fmaxf(tz.x, f.tmin));
    const float exit = min3f(tx.y, ty.y, fminf(tz.y, hl));
    sgn[c] = fword(exit - entry);
  }
  // sign bytes in slot order (byte c of s_lo | s_hi << 32: slot c); slot 7 reads as rejected
  // when the node has fewer than 8 children, as it then stands for the permutation's unused
  // positions (nibble 15: slot 7's sign replicated)
  const uint32_t s_lo = prmt(prmt(sgn[0], sgn[1], 0x0073u), prmt(sgn[2], sgn[3], 0x0073u), 0x5410u);
  const uint32_t s_hi = prmt(prmt(sgn[4], sgn[5], 0x0073u), prmt(sgn[6], sgn[7], 0x0073u), 0x5410u) |
                        ((hd.w - 0x08000000u) & 0x80000000u);
  // bit 8j + 7 of m: the child at visit position j is kept
  const uint64_t m = (uint64_t(~prmt(s_lo, s_hi, perm >> 16) & 0x80808080u) << 32) |
                     (~prmt(s_lo, s_hi, perm & 0xFFFFu) & 0x80808080u);
  if (COUNT) {
    cnt->node[KIND] += 1;
    cnt->box[KIND] += hd.w >> 24;
  }
  // The builder bounds the stack: the entries below this node plus its children minus one
  // never exceed the image's stack size, which the capacity covers.  Checked once per node.
  if (tv.sp + (hd.w >> 24) > sk.cap + 1) {
    flag_error(err, kErrStack);
    tv.walk = false;
    return;
  }
  if (m == 0) {
    wtrav_pop(tv, sk, tid);
    return;
  }
  for (uint64_t rest = m & (m - 1); rest != 0;) {  // all kept but the first, last first
    const int bit = msb64(rest);
    const uint32_t slot = (perm >> ((bit >> 3) * 4)) & 7u;
    sk.ref[tv.sp * sk.stride + tid] = pick8(ra, rb, slot);
    ++tv.sp;
    rest ^= uint64_t(1) << bit;
  }
  const uint32_t slot = (perm >> (((ffs64(m) - 1) >> 3) * 4)) & 7u;
  tv.cur = pick8(ra, rb, slot);
}

// Walks wide nodes until the ray has a leaf record to process (tv.post) or nothing left.
template <int KIND, bool COUNT>
BZR_HD void wtrav_to_leaf(const KindView &K, const RayW &f, float hl, Trav &tv, const Stack &sk,
                          uint32_t tid, uint32_t *err, Counts *cnt) {
  const unsigned lanes = active_lanes();
  for (;;) {
    wtrav_postpone(tv, sk, tid);
    const bool at_node = tv.walk && !(tv.cur & kLeafBit);
    const bool searching = at_node && tv.post == kNoLeaf;
    if (!(COUNT ? searching : warp_any(lanes, searching))) break;
    if (at_node) wtrav_node<KIND, COUNT>(K, f, hl, tv, sk, tid, err, cnt);
  }
  if (tv.post == kNoLeaf && !tv.walk) tv.live = false;  // nothing left to process
}

// The first postponed leaf record: the exact FP64 test of the leaf's box, then its primitives in
// the reference's stored order (blazert/bvh/intersect.h:67-78); the queue moves up by one.  The
// walk then resumes at tv.cur.
template <int KIND, bool COUNT>
BZR_HD void wtrav_leaf(const KindView &K, const Ray &r, const RayW &f, KState &st, float &hl,
                       Trav &tv, const Stack &sk, uint32_t tid, uint32_t *err, Counts *cnt) {
  (void)sk;
  (void)tid;
  constexpr uint32_t kUnits = KIND == kMesh ? 1u : uint32_t(kPayloadDoubles[KIND] / 2);
  if (tv.post == kNoLeaf) return;
  const uint32_t off = tv.post & kIdMask;
  tv.post = tv.post2;
  tv.post2 = kNoLeaf;
  if (uint64_t(off) + kLeafHeaderBytes / 16 > K.n_leaf16) {
    flag_error(err, kErrPrimIndex);
    tv.live = false;
    return;
  }
  const double *L = K.leaves + 2 * size_t(off);
  const double2 px = ld2(L), py = ld2(L + 2), pz = ld2(L + 4);
  const uint4 hdr = ldg(reinterpret_cast<const uint4 *>(L + 6));
  if (COUNT) cnt->leaf[KIND] += 1;
  double key;
  if (box_test(px, py, pz, r, key) && !(key > st.hit)) {
    if (uint64_t(off) + kLeafHeaderBytes / 16 + uint64_t(kUnits) * hdr.y > K.n_leaf16 ||
        uint64_t(hdr.x) + hdr.y > K.n_prims) {
      flag_error(err, kErrPrimIndex);
      tv.live = false;
      return;
    }
    const double before = st.hit;
    for (uint32_t j = 0; j < hdr.y; ++j) {
      const uint32_t pos = hdr.x + j;
      const double *P = L + kLeafHeaderBytes / 8 + size_t(j) * kUnits * 2;
      if (COUNT) cnt->prim[KIND] += 1;
      bool h;
      if (KIND == kMesh)
        h = isect_triangle<false>(K.verts, ldg(reinterpret_cast<const uint4 *>(P)), pos, r, st);
      else if (KIND == kSpheres)
        h = isect_sphere(P, pos, r, st);
      else
        h = isect_plane(P, pos, r, st);
      if (h && r.any_hit) {  // the first hit ends the leaf and the traversal
        tv.live = false;
        return;
      }
    }
    if (st.hit != before) hl = hit_bound(st.hit);
  }
  if (!tv.walk && tv.post == kNoLeaf) tv.live = false;
}

// The end of a wide walk: the barycentrics of a triangle hit, which the walk does not keep.
template <int KIND>
BZR_HD void wtrav_end(const KindView &K, const Ray &r, KState &st) {
  if (KIND == kMesh && st.pos != 0xFFFFFFFFu) tri_uv(K, r, st);
}

// Whole traversal of one kind in mixed precision (the FP64 traversal for cylinders, kinds
// without a wide image and rays the FP32 test does not cover).
template <int KIND, bool COUNT>
BZR_HD bool traverse_mixed(const KindView &K, const Ray &r, KState &st, const Stack &sk,
                           uint32_t tid, uint32_t *err, Counts *cnt) {
  if constexpr (KIND == kCylinders) {
    return traverse<KIND, COUNT>(K, r, st, sk, tid, err, cnt);
  } else {
    const RayW f = make_ray_w(r);
    if (!(K.mixed_ok && f.ok)) return traverse<KIND, COUNT>(K, r, st, sk, tid, err, cnt);
    Trav tv;
    float hl;
    wtrav_begin<KIND, COUNT>(K, r, f, st, hl, tv, cnt);
    while (tv.live) {
      wtrav_to_leaf<KIND, COUNT>(K, f, hl, tv, sk, tid, err, cnt);
      while (tv.live && tv.post != kNoLeaf)
        wtrav_leaf<KIND, COUNT>(K, r, f, st, hl, tv, sk, tid, err, cnt);
    }
    wtrav_end<KIND>(K, r, st);
    return st.hit < r.tmax;
  }
}

struct Best {
  double t, u, v;
  D3 n;
  uint32_t prim, geom;
  bool hit;
};

// post_traversal (trimesh.h:133-143, sphere.h:107-114, plane.h:153-159, cylinder.h:154-160)
template <int KIND>
BZR_HD void take(const SceneView &S, const Ray &r, const KState &st,
                                     Best &best) {
  const KindView &K = S.k[KIND];
  best.t = st.hit;
  best.u = st.u;
  best.v = st.v;
  best.geom = K.geom_id;
  best.hit = true;
  if (KIND == kMesh) {
    // the triangle's words give its id and its vertices, whose normals are stored in the
    // vertices' numbering: one dependent load before the normals
    const uint4 w4 = ldg(reinterpret_cast<const uint4 *>(K.tri) + st.pos);
    best.prim = w4.w & kIdMask;
    auto vn = [&](uint32_t j) { return ld_d4xyz(K.vnorm + kVertexDoubles * size_t(j)); };
    const D3 n0 = vn(w4.x), n1 = vn(w4.y), n2 = vn(w4.z);
    const double w = (1.0 - st.u) - st.v;
    best.n = normalize(add(add(mul(n0, w), mul(n1, st.u)), mul(n2, st.v)));
  } else if (KIND == kSpheres) {
    best.prim = ldg(K.prim_ids + st.pos) & kIdMask;
    const double *P = K.payload + size_t(st.pos) * kPayloadDoubles[kSpheres];
    const D3 c = d3(ldg(P), ldg(P + 1), ldg(P + 2));
    best.n = normalize(sub(add(r.o, mul(r.d, st.hit)), c));
  } else {
    best.prim = ldg(K.prim_ids + st.pos) & kIdMask;
    best.n = normalize(st.n);
  }
}

// Merge of one kind's result into the output record of ray i (blazert/scene.h:161-210): the
// first kind traced writes the whole record (a miss writes the RayHit defaults); later kinds
// overwrite it only when they hit strictly closer -- except triangles, which are always traced
// first and copy unconditionally.  post_traversal supplies the normal.
template <int KIND>
BZR_HD void finalize_kind(const SceneView &S, const Ray &r, const KState &st, uint64_t i,
                          bool first, double *t, double *uv, double *normal, uint32_t *prim,
                          uint32_t *geom, uint8_t *hit) {
  const bool hit_k = st.hit < r.tmax;
  const double prev = first ? 1.7976931348623157e308 : t[i];
  if (hit_k && (KIND == kMesh || st.hit < prev)) {
    Best b;
    take<KIND>(S, r, st, b);
    t[i] = b.t;
    if (uv) {
      uv[2 * i] = b.u;
      uv[2 * i + 1] = b.v;
    }
    if (normal) {
      normal[3 * i] = b.n.x;
      normal[3 * i + 1] = b.n.y;
      normal[3 * i + 2] = b.n.z;
    }
    if (prim) prim[i] = b.prim;
    if (geom) geom[i] = b.geom;
    if (hit) hit[i] = 1;
  } else if (first) {
    t[i] = 1.7976931348623157e308;
    if (uv) uv[2 * i] = uv[2 * i + 1] = 0.0;
    if (normal) normal[3 * i] = normal[3 * i + 1] = normal[3 * i + 2] = 0.0;
    if (prim) prim[i] = 0xFFFFFFFFu;
    if (geom) geom[i] = 0xFFFFFFFFu;
    if (hit) hit[i] = 0;
  }
}

}  // namespace bzr
