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

BZR_HD D3 ld_vertex(const double *verts, uint32_t i) {
  const double *p = verts + size_t(i) * kVertexDoubles;
  const double2 xy = ld2(p), z0 = ld2(p + 2);
  return d3(xy.x, xy.y, z0.x);
}

// blazert/primitives/trimesh.h:153-181.  F holds the triangle's three vertex indices; v0,
// e1 = v0 - v1, e2 = v2 - v0 (the reference Triangle's members, trimesh.h:19-31) and
// n = cross(e1, e2) are formed here with the reference's operations, hence the same bits.
BZR_HD bool isect_triangle(const double *verts, uint4 F, uint32_t pos, const Ray &r,
                           KState &st) {
  const D3 v0 = ld_vertex(verts, F.x), v1 = ld_vertex(verts, F.y), v2 = ld_vertex(verts, F.z);
  const D3 e1 = sub(v0, v1), e2 = sub(v2, v0);
  const D3 n = cross(e1, e2);
  const D3 c = sub(v0, r.o);
  const D3 rr = cross(r.d, c);
  const double det = dot(n, r.d);
  const double abs_det = fabs(det);
  const double u = product_sign(dot(rr, e2), det);
  const double v = product_sign(dot(rr, e1), det);
  const double w = (abs_det - u) - v;
  if (u >= -kTol && v >= -kTol && w >= -kTol) {
    const double t = product_sign(dot(n, c), det);
    if (t >= abs_det * r.tmin && abs_det * st.hit > t) {
      const double inv_det = 1.0 / abs_det;
      st.hit = t * inv_det;
      st.u = u * inv_det;
      st.v = v * inv_det;
      st.pos = pos;
      return true;
    }
  }
  return false;
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

// Traversal stack in shared memory, entry j of thread t at [j * blockDim.x + t].
struct Stack {
  double *key;
  uint32_t *ref;
  uint32_t cap, stride;
};

// Work counters of one ray (counting kernels only): per kind the box tests (the reference's
// node pops: the root plus both children of every accepted internal node) and primitive tests.
struct Counts {
  uint32_t box[kNumKinds];
  uint32_t prim[kNumKinds];
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
};

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
    const double *nd = K.nodes64 + size_t(tv.cur) * kNode64Doubles;
    const double2 a0 = ld2(nd), a1 = ld2(nd + 2), a2 = ld2(nd + 4);
    const double2 b0 = ld2(nd + 6), b1 = ld2(nd + 8), b2 = ld2(nd + 10);
    const uint4 meta = ldg(reinterpret_cast<const uint4 *>(nd + 12));
    double k0, k1;
    if (COUNT) cnt->box[KIND] += 2;
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
// Mixed precision (BZR_MODE_MIXED): slab tests in FP32 on the 64-byte nodes, with every
// decision equal to the FP64 one.
//
// For an eligible ray, every FP32 entry/exit distance a32 = (fl32(plane) - fl32(o)) * fl32(inv)
// is within delta of the FP64 value of the reference's slab test:
//   |a32 - a64| <= 2^-21 * max|inv| * (coord_max + max|o|)  (+ tiny absolute terms),
// from the relative errors of the five FP32 roundings (<= 3 * 2^-23 in all) and the FP64 ones
// (l1 = 1 + 2^-50 included).  A child is accepted or rejected in FP32 only when the FP32
// comparison holds with that margin (sums rounded outward); otherwise its exact FP64 test
// runs on the FP64 node.  The pop-time comparison of the entry distance with the hit distance
// is decided the same way, re-testing the child in FP64 when it falls inside the margin.  So
// the accepted nodes, and hence the leaves, primitive tests and results, are exactly the FP64
// path's.  Rays that are not eligible (a zero, tiny or non-finite direction component, huge
// coordinates, non-finite tmin, NaN tmax) and kinds with a non-finite box use the FP64 path.
struct RayF {
  float o[3], inv[3];
  float tmin, delta;
  bool ok;
};

BZR_HD float fadd_up(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fadd_ru(a, b);
#else
  return nextafterf(float(double(a) + double(b)), __builtin_inff());  // conservative
#endif
}
BZR_HD float fadd_down(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fadd_rd(a, b);
#else
  return nextafterf(float(double(a) + double(b)), -__builtin_inff());
#endif
}

BZR_HD RayF make_ray_f(const Ray &r, float coord_max) {
  RayF f;
  const double inv[3] = {r.inv.x, r.inv.y, r.inv.z}, o[3] = {r.o.x, r.o.y, r.o.z};
  double imax = 0.0, imin = 1e300, omax = 0.0;
  bool ok = isfinite(r.tmin) && !isnan(r.tmax) && isfinite(coord_max) &&
            coord_max <= 1e18f;
  for (int a = 0; a < 3; ++a) {
    const double ai = fabs(inv[a]);
    ok = ok && isfinite(inv[a]) && ai > 0.0 && isfinite(o[a]) && fabs(o[a]) <= 1e18;
    imax = ai > imax ? ai : imax;
    imin = ai < imin ? ai : imin;
    omax = fabs(o[a]) > omax ? fabs(o[a]) : omax;
    f.o[a] = float(o[a]);
    f.inv[a] = float(inv[a]);
  }
  ok = ok && imax <= 16384.0 * imin && imax <= 1e18;
  const double d = 4.76837158203125e-07 /* 2^-21 */ * (imax * (double(coord_max) + omax) + fabs(r.tmin)) +
                   1e-30 * (1.0 + imax);
  f.tmin = float(r.tmin);
  f.delta = ok ? nextafterf(float(d), __builtin_inff()) : 0.0f;
  f.ok = ok && isfinite(f.delta);
  return f;
}

// FP32 slab test of one box given as (lo, hi) pairs per axis: 1 accept for some hit distance,
// 0 reject for every hit distance, 2 undecided in FP32.  mn receives the FP32 entry distance.
BZR_HD int box_test32(float lx, float hx, float ly, float hy, float lz, float hz, const RayF &f,
                      const Ray &r, float &mn) {
  const float ax = ((r.sx ? hx : lx) - f.o[0]) * f.inv[0];
  const float bx = ((r.sx ? lx : hx) - f.o[0]) * f.inv[0];
  const float ay = ((r.sy ? hy : ly) - f.o[1]) * f.inv[1];
  const float by = ((r.sy ? ly : hy) - f.o[1]) * f.inv[1];
  const float az = ((r.sz ? hz : lz) - f.o[2]) * f.inv[2];
  const float bz = ((r.sz ? lz : hz) - f.o[2]) * f.inv[2];
  mn = fmaxf(fmaxf(f.tmin, ax), fmaxf(ay, az));
  const float ex = fminf(fminf(bx, by), bz);
  if (fadd_up(mn, f.delta) <= fadd_down(ex, -f.delta)) return 1;
  if (fadd_down(mn, -f.delta) > fadd_up(ex, f.delta)) return 0;
  return 2;
}

// Exact FP64 slab test of child `slot` of FP64 node `node`.
BZR_HD bool child_test64(const KindView &K, uint32_t node, int slot, const Ray &r, double &key) {
  const double *nd = K.nodes64 + size_t(node) * kNode64Doubles + 6 * slot;
  return box_test(ld2(nd), ld2(nd + 2), ld2(nd + 4), r, key);
}

// Mixed stack entry: ref in sk.ref; the key slot holds {float key, uint32 aux} with
// aux = parent << 2 | slot << 1 | exact.  exact: key is fl32 of the FP64 entry distance.
BZR_HD void push32(const Stack &sk, uint32_t tid, uint32_t sp, uint32_t ref, float key,
                   uint32_t aux) {
  uint32_t *w = reinterpret_cast<uint32_t *>(sk.key + sp * sk.stride + tid);
  float kk = key;
  uint32_t kb;
  std::memcpy(&kb, &kk, 4);
  w[0] = kb;
  w[1] = aux;
  sk.ref[sp * sk.stride + tid] = ref;
}

// Pop-time decision !(key64 > h) from the FP32 key and its margin; -1 when undecided.
BZR_HD int key_decide(float key, float margin, double h) {
  if (double(fadd_up(key, margin)) <= h) return 1;
  if (double(fadd_down(key, -margin)) > h) return 0;
  return -1;
}
BZR_HD float exact_margin(float key) {
  return nextafterf(fabsf(key) * 1.1920928955078125e-07f, __builtin_inff()) + 1.4e-45f;
}

template <int KIND>
BZR_HD void trav_pop32(const KindView &K, const Ray &r, const RayF &f, Trav &tv, const KState &st,
                       const Stack &sk, uint32_t tid) {
  while (tv.sp > 0) {
    --tv.sp;
    const uint32_t *w = reinterpret_cast<const uint32_t *>(sk.key + tv.sp * sk.stride + tid);
    const uint32_t kb = w[0], aux = w[1];
    float key;
    std::memcpy(&key, &kb, 4);
    int d = key_decide(key, (aux & 1u) ? exact_margin(key) : f.delta, st.hit);
    if (d < 0) {
      double k64;
      child_test64(K, aux >> 2, int((aux >> 1) & 1u), r, k64);
      d = !(k64 > st.hit);
    }
    if (d) {
      tv.cur = sk.ref[tv.sp * sk.stride + tid];
      return;
    }
  }
  tv.live = false;
}

template <int KIND, bool COUNT>
BZR_HD void trav_to_leaf32(const KindView &K, const Ray &r, const RayF &f, const KState &st,
                           Trav &tv, const Stack &sk, uint32_t tid, uint32_t *err, Counts *cnt) {
  while (tv.live && !(tv.cur & kLeafBit)) {
    if (tv.cur >= K.n_internal) {
      flag_error(err, kErrNodeIndex);
      tv.live = false;
      return;
    }
    const float *nf = K.nodes32 + size_t(tv.cur) * kNode32Floats;
    const float4 q0 = ldg(reinterpret_cast<const float4 *>(nf));
    const float4 q1 = ldg(reinterpret_cast<const float4 *>(nf + 4));
    const float4 q2 = ldg(reinterpret_cast<const float4 *>(nf + 8));
    const uint4 meta = ldg(reinterpret_cast<const uint4 *>(nf + 12));
    if (COUNT) cnt->box[KIND] += 2;
    float m0, m1;
    int d0 = box_test32(q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, f, r, m0);
    int d1 = box_test32(q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, f, r, m1);
    bool e0 = false, e1 = false;
    double k0 = 0.0, k1 = 0.0;
    if (d0 == 2) {
      d0 = child_test64(K, tv.cur, 0, r, k0) ? 1 : 0;
      e0 = true;
    }
    if (d1 == 2) {
      d1 = child_test64(K, tv.cur, 1, r, k1) ? 1 : 0;
      e1 = true;
    }
    const unsigned near = meta.z == 0 ? r.sx : (meta.z == 1 ? r.sy : r.sz);
    const int dn = near ? d1 : d0, df = near ? d0 : d1;
    const bool en = near ? e1 : e0, ef = near ? e0 : e1;
    const double kn = near ? k1 : k0, kf = near ? k0 : k1;
    const float mnn = near ? m1 : m0, mnf = near ? m0 : m1;
    const uint32_t rn = near ? meta.y : meta.x, rf = near ? meta.x : meta.y;
    if (df) {
      if (tv.sp >= sk.cap) {
        flag_error(err, kErrStack);
        tv.live = false;
        return;
      }
      push32(sk, tid, tv.sp, rf, ef ? float(kf) : mnf,
             (tv.cur << 2) | ((near ? 0u : 1u) << 1) | (ef ? 1u : 0u));
      ++tv.sp;
    }
    bool take_near = false;
    if (dn) {
      if (en) {
        take_near = !(kn > st.hit);
      } else {
        const int d = key_decide(mnn, f.delta, st.hit);
        if (d >= 0) {
          take_near = d;
        } else {
          double k;
          child_test64(K, tv.cur, int(near), r, k);
          take_near = !(k > st.hit);
        }
      }
    }
    if (take_near) {
      tv.cur = rn;
    } else {
      trav_pop32<KIND>(K, r, f, tv, st, sk, tid);
    }
  }
}

template <int KIND, bool COUNT>
BZR_HD void trav_leaf32(const KindView &K, const Ray &r, const RayF &f, KState &st, Trav &tv,
                        const Stack &sk, uint32_t tid, uint32_t *err, Counts *cnt) {
  uint32_t pos = tv.cur & kIdMask;
  for (;;) {
    if (pos >= K.n_prims) {
      flag_error(err, kErrPrimIndex);
      tv.live = false;
      return;
    }
    if (COUNT) cnt->prim[KIND] += 1;
    bool h;
    const uint32_t id = isect<KIND>(K, pos, r, st, h);
    if (h && r.any_hit) {
      tv.live = false;
      return;
    }
    if (id & kLastBit) break;
    ++pos;
  }
  trav_pop32<KIND>(K, r, f, tv, st, sk, tid);
}

// Whole traversal of one kind in mixed precision (FP64 for rays or kinds not eligible).
template <int KIND, bool COUNT>
BZR_HD bool traverse_mixed(const KindView &K, const Ray &r, KState &st, const Stack &sk,
                           uint32_t tid, uint32_t *err, Counts *cnt) {
  const RayF f = make_ray_f(r, K.coord_max);
  if (!(K.mixed_ok && f.ok)) return traverse<KIND, COUNT>(K, r, st, sk, tid, err, cnt);
  Trav tv;
  trav_begin<KIND, COUNT>(K, r, st, tv, cnt);
  while (tv.live) {
    trav_to_leaf32<KIND, COUNT>(K, r, f, st, tv, sk, tid, err, cnt);
    if (tv.live) trav_leaf32<KIND, COUNT>(K, r, f, st, tv, sk, tid, err, cnt);
  }
  return st.hit < r.tmax;
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
  best.prim = ldg(K.prim_ids + st.pos) & kIdMask;
  best.geom = K.geom_id;
  best.hit = true;
  if (KIND == kMesh) {
    const uint32_t *F = S.faces + 3 * size_t(best.prim);
    const uint32_t f0 = ldg(F), f1 = ldg(F + 1), f2 = ldg(F + 2);
    const D3 n0 = d3(ldg(S.vert_n + 3 * f0), ldg(S.vert_n + 3 * f0 + 1),
                     ldg(S.vert_n + 3 * f0 + 2));
    const D3 n1 = d3(ldg(S.vert_n + 3 * f1), ldg(S.vert_n + 3 * f1 + 1),
                     ldg(S.vert_n + 3 * f1 + 2));
    const D3 n2 = d3(ldg(S.vert_n + 3 * f2), ldg(S.vert_n + 3 * f2 + 1),
                     ldg(S.vert_n + 3 * f2 + 2));
    const double w = (1.0 - st.u) - st.v;
    best.n = normalize(add(add(mul(n0, w), mul(n1, st.u)), mul(n2, st.v)));
  } else if (KIND == kSpheres) {
    const double *P = K.payload + size_t(st.pos) * kPayloadDoubles[kSpheres];
    const D3 c = d3(ldg(P), ldg(P + 1), ldg(P + 2));
    best.n = normalize(sub(add(r.o, mul(r.d, st.hit)), c));
  } else {
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
