// Point-to-primitive distances, shared by the sm_100a kernel (distance.cu) and, compiled as host
// code, by the test-only CPU emulator (tests/emu/).  Each function restates the reference's
// distance_to_surface for one primitive kind in the reference's own operation order (the blaze
// operations as the oracle's shim defines them: dot = (x0*y0 + x1*y1) + x2*y2, M * v row by row
// in the same order, element-wise vector arithmetic), compiled without contraction
// (--fmad=false / -ffp-contract=off), so that the results equal the reference's bit for bit:
// sqrt and division are correctly rounded on both sides.
//
//   sphere    blazert/primitives/sphere.h:179-182
//   plane     blazert/primitives/plane.h:272-284 (the in-rectangle test compares the LOCAL
//             point with the plane's WORLD centre, as the reference does; outside it the
//             distance is DBL_MAX)
//   cylinder  blazert/primitives/cylinder.h:677-759 with the ellipse search of
//             cylinder.h:498-673 (Newton iterations on the closest point of the ellipse)
//   triangle  closest_point_on_triangle, blazert/primitives/trimesh_distance.h:177-218 (Eberly's
//             region method) on the face's vertices v0, v1, v2, and the distance
//             norm(closest - point).  The reference's own triangle distance_to_surface
//             (trimesh.h:183-192) cannot be instantiated: it returns a vector as a scalar and
//             rebuilds v1, v2 from the stored edges with the wrong signs.
#pragma once
#include "trace_core.cuh"

namespace bzr {

constexpr double kDblEps = 2.220446049250313080847e-16;  // std::numeric_limits<double>::epsilon()

// payload_doubles(kind) in device code
BZR_HD int payload_doubles(int kind) {
  return kind == kSpheres ? 4 : kind == kPlanes ? 14 : kind == kCylinders ? 16 : 0;
}

// std::min(a, b) and std::min({...}): the first argument unless a later one is strictly less.
BZR_HD double min_first(double a, double b) { return b < a ? b : a; }

// local = trans(R) * (p - c) with R row-major: local[i] = (R(0,i) v0 + R(1,i) v1) + R(2,i) v2.
BZR_HD D3 to_local(const double *R, D3 c, D3 p) {
  const D3 v = sub(p, c);
  return {(R[0] * v.x + R[3] * v.y) + R[6] * v.z, (R[1] * v.x + R[4] * v.y) + R[7] * v.z,
          (R[2] * v.x + R[5] * v.y) + R[8] * v.z};
}

// sphere.h:179-182: |norm(center - point) - radius|
BZR_HD double sphere_distance(D3 c, double r, D3 p) { return fabs(norm(sub(c, p)) - r); }

// plane.h:272-284
BZR_HD double plane_distance(D3 c, double dxs, double dys, const double *R, D3 p) {
  const D3 lp = to_local(R, c, p);
  const double dx = dxs / 2, dy = dys / 2;
  const double cx = c.x, cy = c.y;
  if ((lp.x >= cx - dx) && (lp.x <= cx + dx) && (lp.y >= cy - dy) && (lp.y <= cy + dy))
    return fabs(lp.z);
  return kDblMax;
}

// The four branches of the ellipse search (cylinder.h:512-599).  UPPER/LOWER half plane,
// iterating over X or Y.
enum EllipseBranch : int { kUpperX = 0, kLowerX = 1, kUpperY = 2, kLowerY = 3 };

// sqrt(|val^2 - s^2|) as the reference forms it: the larger square first
BZR_HD double root_gap(double val, double s) {
  return (val * val > s * s) ? sqrt(val * val - s * s) : sqrt(s * s - val * val);
}

// distance_derivative (cylinder.h:516-547): R'(val)
template <int BR>
BZR_HD double ellipse_derivative(double a, double b, double xq, double yq, double val) {
  if (BR == kUpperX) {
    const double s = root_gap(val, a);
    return -2 * (xq - val) - 2 * b * val * (b / a * s - yq) / (a * s);
  } else if (BR == kLowerX) {
    const double s = root_gap(val, a);
    return -2 * (xq - val) - 2 * b * val * (b / a * s + yq) / (a * s);
  } else if (BR == kUpperY) {
    const double s = root_gap(val, b);
    return -2 * (yq - val) - 2 * a * val * (a / b * s + xq) / (b * s);
  } else {
    const double s = root_gap(val, b);
    return -2 * (yq - val) - 2 * a * val * (a / b * s - xq) / (b * s);
  }
}

// single_newton_iteration (cylinder.h:551-590): val - R'(val) / R''(val) in closed form
template <int BR>
BZR_HD double ellipse_newton_step(double a, double b, double xq, double yq, double val) {
  if (BR == kUpperX) {
    const double s = root_gap(val, a);
    return ((a * a * a * xq - a * val * val * xq) * s + b * val * val * val * yq) /
           ((a * a * a - a * b * b - a * val * val + b * b * val * val / a) * s + a * a * b * yq);
  } else if (BR == kLowerX) {
    const double s = root_gap(val, a);
    return ((-a * a * a * xq + a * val * val * xq) * s + b * val * val * val * yq) /
           ((-a * a * a + a * b * b + a * val * val - b * b * val * val / a) * s + a * a * b * yq);
  } else if (BR == kUpperY) {
    const double s = root_gap(val, b);
    return ((b * b * b * yq - b * val * val * yq) * s + a * val * val * val * xq) /
           ((b * b * b - b * a * a - b * val * val + a * a * val * val / b) * s + b * b * a * xq);
  } else {
    const double s = root_gap(val, b);
    return ((-b * b * b * yq + b * val * val * yq) * s + a * val * val * val * xq) /
           ((-b * b * b + b * a * a + b * val * val - a * a * val * val / b) * s + b * b * a * xq);
  }
}

// newton_iteration (cylinder.h:594-614): at most 100 steps while |R'| >= 1e-7; a value that
// lands on |val| == a is nudged by one epsilon (against a in every branch, as the reference).
template <int BR>
BZR_HD double ellipse_newton(double a, double b, double xq, double yq, double val0) {
  double cnt = 0;
  while ((fabs(ellipse_derivative<BR>(a, b, xq, yq, val0)) >= 1e-7) && (cnt < 100)) {
    const double val = ellipse_newton_step<BR>(a, b, xq, yq, val0);
    val0 = val;
    cnt++;
    if (fabs(val0) == a) val0 += kDblEps;
  }
  return val0;
}

// find_minimum_distance_to_ellipse (cylinder.h:622-673): the shortest distance from (xq, yq)
// to the ellipse x^2/a^2 + y^2/b^2 = 1, by the branch the point's sector selects.
BZR_HD double ellipse_distance(double a, double b, double xq, double yq) {
  const double percentage = 0.95;
  if (((xq >= 0) && (yq >= (b / a) * xq)) || ((xq <= 0) && (yq >= (-b / a) * xq))) {
    const double x0 = xq > 0 ? percentage * a : -percentage * a;
    const double x_min = ellipse_newton<kUpperX>(a, b, xq, yq, x0);
    const double s = sqrt(a * a - x_min * x_min);
    const double y_min = b / a * s;
    return sqrt((xq - x_min) * (xq - x_min) + (yq - y_min) * (yq - y_min));
  } else if (((xq >= 0) && (yq <= (-b / a) * xq)) || ((xq <= 0) && (yq <= (b / a) * xq))) {
    const double x0 = xq > 0 ? percentage * a : -percentage * a;
    const double x_min = ellipse_newton<kLowerX>(a, b, xq, yq, x0);
    const double s = sqrt(a * a - x_min * x_min);
    const double y_min = -b / a * s;
    return sqrt((xq - x_min) * (xq - x_min) + (yq - y_min) * (yq - y_min));
  } else if ((xq >= 0) && (yq <= (b / a) * xq) && (yq >= (-b / a) * xq)) {
    const double y0 = yq > 0 ? percentage * b : -percentage * b;
    const double y_min = ellipse_newton<kUpperY>(a, b, xq, yq, y0);
    const double s = sqrt(b * b - y_min * y_min);
    const double x_min = a / b * s;
    return sqrt((yq - y_min) * (yq - y_min) + (xq - x_min) * (xq - x_min));
  } else {
    const double y0 = yq > 0 ? percentage * b : -percentage * b;
    const double y_min = ellipse_newton<kLowerY>(a, b, xq, yq, y0);
    const double s = sqrt(b * b - y_min * y_min);
    const double x_min = -a / b * s;
    return sqrt((yq - y_min) * (yq - y_min) + (xq - x_min) * (xq - x_min));
  }
}

// cylinder.h:677-759
BZR_HD double cylinder_distance(D3 c, double a, double b, double height, const double *R,
                                D3 p) {
  const D3 lp = to_local(R, c, p);
  const double dist_top = fabs(lp.z - height / 2);
  const double dist_bottom = fabs(lp.z + height / 2);
  const double x_q = lp.x, y_q = lp.y, z_q = lp.z;
  if (x_q == 0 && y_q == 0) {  // isZero(point_xy)
    if ((z_q > height / 2) || (z_q < -height / 2)) return min_first(dist_top, dist_bottom);
    return min_first(min_first(min_first(a, b), dist_top), dist_bottom);
  }
  const double ellipse = (x_q * x_q) / (a * a) + (y_q * y_q) / (b * b) - 1;
  if (fabs(ellipse) < kDblEps) {
    if ((z_q > height / 2) || (z_q < -height / 2)) return min_first(dist_top, dist_bottom);
    return 0.0;
  }
  if (ellipse < 0) {
    if (z_q >= height / 2) return dist_top;
    if (z_q <= -height / 2) return dist_bottom;
    const double dist_shell = ellipse_distance(a, b, x_q, y_q);
    return min_first(min_first(dist_shell, dist_bottom), dist_top);
  }
  if (ellipse > 0) {
    const double dist_shell = ellipse_distance(a, b, x_q, y_q);
    if ((z_q < height / 2) && (z_q > -height / 2)) return dist_shell;
    const double dist1 = sqrt(dist_shell * dist_shell + dist_top * dist_top);
    const double dist2 = sqrt(dist_shell * dist_shell + dist_bottom * dist_bottom);
    return min_first(dist1, dist2);
  }
  return -1.0;  // a NaN ellipse value (degenerate semi-axes)
}

// trimesh_distance.h:177-218 with the region helpers r0..r6 (:37-163)
BZR_HD D3 closest_point_on_triangle(D3 v0, D3 v1, D3 v2, D3 p) {
  const D3 E0 = sub(v1, v0), E1 = sub(v2, v0), D = sub(v0, p);
  const double a = dot(E0, E0), b = dot(E0, E1), c = dot(E1, E1);
  const double d = dot(E0, D), e = dot(E1, D);
  const double det = a * c - b * b;
  double s = b * e - c * d;
  double t = b * d - a * e;
  if (s + t <= det) {
    if (s < 0.0) {
      if (t < 0.0) {  // region 4
        if (d < 0.0) {
          t = 0.0;
          s = (-d >= a) ? 1.0 : -d / a;
        } else {
          s = 0.0;
          t = (e >= 0.0) ? 0.0 : ((-e >= c) ? 1.0 : -e / c);
        }
      } else {  // region 3
        s = 0.0;
        t = (e >= 0.0) ? 0.0 : ((-e >= c) ? 1.0 : -e / c);
      }
    } else if (t < 0.0) {  // region 5
      t = 0.0;
      s = (d >= 0.0) ? 0.0 : ((-d >= a) ? 1.0 : -d / a);
    } else {  // region 0
      const double inv_det = 1.0 / det;
      s *= inv_det;
      t *= inv_det;
    }
  } else {
    if (s < 0.0) {  // region 2
      const double tmp0 = b + d, tmp1 = c + e;
      if (tmp1 > tmp0) {
        const double numer = tmp1 - tmp0, denom = a - 2.0 * b + c;
        s = (numer >= denom) ? 1.0 : numer / denom;
        t = 1.0 - s;
      } else {
        s = 0.0;
        t = (tmp1 <= 0.0) ? 1.0 : ((e >= 0.0) ? 0.0 : -e / c);
      }
    } else if (t < 0.0) {  // region 6
      const double tmp0 = b + e, tmp1 = a + d;
      if (tmp1 > tmp0) {
        const double numer = tmp1 - tmp0, denom = a - 2.0 * b + c;
        t = (numer >= denom) ? 1.0 : numer / denom;
        s = 1.0 - t;
      } else {
        t = 0.0;
        s = (tmp1 <= 0.0) ? 1.0 : ((d >= 0.0) ? 0.0 : -d / a);
      }
    } else {  // region 1
      const double numer = c + e - b - d;
      if (numer <= 0.0) {
        s = 0.0;
      } else {
        const double denom = a - 2.0 * b + c;
        s = (numer >= denom) ? 1.0 : numer / denom;
      }
      t = 1.0 - s;
    }
  }
  return add(add(v0, mul(E0, s)), mul(E1, t));
}

// Distance from p to the primitive at leaf-ordered position q of kind `kind` (closest point
// too for triangles).
BZR_HD double distance_at(const SceneView &S, int kind, uint32_t q, D3 p, D3 *closest) {
  const KindView &K = S.k[kind];
  if (kind == kMesh) {
    const uint32_t *w = K.tri + 4 * size_t(q);
    D3 v[3];
    for (int j = 0; j < 3; ++j) {
      const double *x = K.verts + size_t(kVertexDoubles) * ldg(w + j);
      v[j] = d3(ldg(x), ldg(x + 1), ldg(x + 2));
    }
    *closest = closest_point_on_triangle(v[0], v[1], v[2], p);
    return norm(sub(*closest, p));
  }
  const double *P = K.payload + size_t(payload_doubles(kind)) * q;
  double r[15];
  for (int j = 0; j < 15; ++j) r[j] = j < payload_doubles(kind) ? ldg(P + j) : 0.0;
  const D3 c = d3(r[0], r[1], r[2]);
  if (kind == kSpheres) return sphere_distance(c, r[3], p);
  if (kind == kPlanes) return plane_distance(c, r[3], r[4], r + 5, p);
  return cylinder_distance(c, r[3], r[4], r[5], r + 6, p);
}

// One query of the per-primitive form: primitive `id` of `kind` and point p.  Returns NaN for
// an id outside the kind (and sets *bad).
BZR_HD double distance_query(const SceneView &S, int kind, uint32_t id, D3 p, D3 *closest,
                             bool *bad) {
  const KindView &K = S.k[kind];
  *bad = id >= K.n_prims;
  if (*bad) {
    const double nan = bitsd(0x7FF8000000000000LL);
    *closest = d3(nan, nan, nan);
    return nan;
  }
  return distance_at(S, kind, ldg(K.pos_of + id), p, closest);
}

// ---------------------------------------------------------------------------------------------
// Scene-level query: the smallest per-primitive distance over every primitive of the scene,
// with the semantics of an exhaustive loop over the kinds in the order triangles, spheres,
// planes, cylinders and, within a kind, over the primitives by increasing id, keeping the first
// strictly smaller value (so NaN values never win, and among equal distances the first kind and
// the lowest id).
//
// Triangles and spheres lie inside their BVH boxes, so their distances are bounded below by the
// distance from p to a box: the query walks those BVHs nearest child first and skips a subtree
// whose box is farther than the best distance plus a margin that covers the rounding of both
// sides (1e-12 of the coordinate scale, thousands of ulps), which keeps the result identical to
// the exhaustive loop.  The reference's plane distance is not bounded by the plane's box (its
// rectangle test mixes local and world coordinates) and a cylinder's box is built from six
// points of the shell that need not enclose it, so those kinds are evaluated exhaustively, a
// cylinder skipped when its bounding ball (radius sqrt(max(a, b)^2 + (h / 2)^2)) is farther
// than the best distance plus the margin.

struct NearestState {
  double best = 0.0;
  uint32_t prim = 0xFFFFFFFFu;
  uint32_t geom = 0xFFFFFFFFu;
  int kind = -1;
};

BZR_HD double distance_margin(double scale, double best) { return 1e-12 * (scale + best); }

BZR_HD void nearest_offer(NearestState &st, int kind, uint32_t geom, uint32_t id, double d) {
  if (d < st.best || (d == st.best && st.kind == kind && id < st.prim)) {
    st.best = d;
    st.prim = id;
    st.geom = geom;
    st.kind = kind;
  }
}

// Distance from p to the box [lo, hi] (0 inside).
BZR_HD double box_distance(const double *lohi_x, const double *lohi_y, const double *lohi_z,
                           D3 p) {
  const double gx = fmax(fmax(lohi_x[0] - p.x, p.x - lohi_x[1]), 0.0);
  const double gy = fmax(fmax(lohi_y[0] - p.y, p.y - lohi_y[1]), 0.0);
  const double gz = fmax(fmax(lohi_z[0] - p.z, p.z - lohi_z[1]), 0.0);
  return sqrt((gx * gx + gy * gy) + gz * gz);
}

BZR_HD void nearest_leaf(const SceneView &S, int kind, uint32_t q, D3 p, NearestState &st) {
  const KindView &K = S.k[kind];
  for (;; ++q) {
    if (q >= K.n_prims) break;  // a malformed leaf reference; the leaf ends here
    const uint32_t w = ldg(K.prim_ids + q);
    D3 c;
    nearest_offer(st, kind, K.geom_id, w & kIdMask, distance_at(S, kind, q, p, &c));
    if (w & kLastBit) break;
  }
}

// Every primitive of the kind in leaf order.
BZR_HD void nearest_all(const SceneView &S, int kind, D3 p, double scale, NearestState &st) {
  const KindView &K = S.k[kind];
  for (uint32_t q = 0; q < K.n_prims; ++q) {
    const uint32_t id = ldg(K.prim_ids + q) & kIdMask;
    if (kind == kCylinders) {
      const double *P = K.payload + size_t(payload_doubles(kind)) * q;
      const double a = ldg(P + 3), b = ldg(P + 4), h2 = ldg(P + 5) / 2;
      const double ab = fmax(a, b);
      const double rb = sqrt(ab * ab + h2 * h2);
      const double gap = norm(sub(d3(ldg(P), ldg(P + 1), ldg(P + 2)), p)) - rb;
      if (gap > st.best + distance_margin(scale + rb, st.best)) continue;
    }
    D3 c;
    nearest_offer(st, kind, K.geom_id, id, distance_at(S, kind, q, p, &c));
  }
}

// Nearest-first walk of one kind's BVH (triangles, spheres).  stack holds cap entries; a tree
// that would need more is evaluated exhaustively instead (only trees deeper than the stack).
BZR_HD void nearest_bvh(const SceneView &S, int kind, D3 p, double scale, NearestState &st,
                        uint32_t *stack_ref, double *stack_key, uint32_t cap) {
  const KindView &K = S.k[kind];
  if (S.stack_cap > cap) {
    nearest_all(S, kind, p, scale, st);
    return;
  }
  const double root = box_distance(K.root_box, K.root_box + 2, K.root_box + 4, p);
  if (root > st.best + distance_margin(scale, st.best)) return;
  uint32_t ref = K.root_ref, sp = 0;
  for (;;) {
    if (ref & kLeafBit) {
      nearest_leaf(S, kind, ref & ~kLeafBit, p, st);
    } else if (ref < K.n_internal) {
      const double *nd = K.nodes64 + size_t(kNode64Doubles) * ref;
      double bx[12];
      for (int j = 0; j < 12; ++j) bx[j] = ldg(nd + j);
      const long long refs = dbits(ldg(nd + 12));  // {ref0, ref1} as the low and high words
      const uint32_t meta[2] = {uint32_t(refs), uint32_t(static_cast<unsigned long long>(refs) >> 32)};
      const double d0 = box_distance(bx, bx + 2, bx + 4, p);
      const double d1 = box_distance(bx + 6, bx + 8, bx + 10, p);
      const double lim = st.best + distance_margin(scale, st.best);
      const bool t0 = !(d0 > lim), t1 = !(d1 > lim);
      if (t0 && t1) {
        const bool first1 = d1 < d0;
        stack_ref[sp] = first1 ? meta[0] : meta[1];
        stack_key[sp] = first1 ? d0 : d1;
        ++sp;
        ref = first1 ? meta[1] : meta[0];
        continue;
      }
      if (t0 || t1) {
        ref = t0 ? meta[0] : meta[1];
        continue;
      }
    }
    bool found = false;
    while (sp > 0) {
      --sp;
      if (!(stack_key[sp] > st.best + distance_margin(scale, st.best))) {
        ref = stack_ref[sp];
        found = true;
        break;
      }
    }
    if (!found) return;
  }
}

BZR_HD NearestState nearest_surface(const SceneView &S, D3 p, uint32_t *stack_ref,
                                    double *stack_key, uint32_t cap) {
  NearestState st;
  st.best = BZR_INF;
  const double ps = fmax(fmax(fabs(p.x), fabs(p.y)), fabs(p.z));
  for (int kind = 0; kind < kNumKinds; ++kind) {
    const KindView &K = S.k[kind];
    if (!K.present || K.n_prims == 0) continue;
    const double scale = ps + double(K.coord_max);
    if (kind == kMesh || kind == kSpheres)
      nearest_bvh(S, kind, p, scale, st, stack_ref, stack_key, cap);
    else
      nearest_all(S, kind, p, scale, st);
  }
  return st;
}

}  // namespace bzr
