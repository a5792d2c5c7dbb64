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
#include <limits>

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

// The ellipse search (cylinder.h:498-673).  The reference has four branches -- the point's
// sector selects the upper or lower half plane and whether the iteration runs over x or y --
// each with its own derivative (distance_derivative, :516-547) and Newton step
// (single_newton_iteration, :551-590).  All four are the same expressions under a renaming,
// and are evaluated here by ONE loop so that the lanes of a warp in different sectors iterate
// together:
//   A, B   the semi-axis of the iterated coordinate and the other one (a, b over x; b, a over y)
//   X, Y   the point's iterated coordinate and the other one
//   sg     +1 upper / -1 lower: the sign of the A^3 terms of the step and of the final other
//          coordinate (-b / a * sqrt in the lower branches)
//   tg     the sign of Y in the derivative's bracket: (B / A * s - tg * Y) -- +1 for upper-x
//          and lower-y, -1 for lower-x and upper-y
// Each operation is the reference's with a sign applied exactly where its expression has one
// (x - (-y) and x + y, (-a) * a and -(a * a) are the same bits), so every branch's values are
// reproduced bit for bit.

// sqrt(|val^2 - s^2|) as the reference forms it: the larger square first
BZR_HD double root_gap(double val, double s) {
  return (val * val > s * s) ? sqrt(val * val - s * s) : sqrt(s * s - val * val);
}

struct EllipseBranch {
  double A, B, X, Y, sg, tg;
};

// The search's loop-invariant sub-expressions, each formed exactly as the reference's
// expression forms it (left to right), so that using them gives the same bits.
struct EllipseSearch {
  EllipseBranch e;
  double BA = 0.0;    // B / A
  double B2 = 0.0;    // 2 * B
  double A3X = 0.0;   // (+-A) * A * A * X
  double D0 = 0.0;    // (+-A) * A * A -+ A * B * B
  double BB = 0.0;    // B * B
  double AABY = 0.0;  // A * A * B * Y
};

BZR_HD EllipseSearch ellipse_search(const EllipseBranch &e) {
  EllipseSearch S;
  S.e = e;
  S.BA = e.B / e.A;
  S.B2 = 2 * e.B;
  S.A3X = (e.sg * e.A) * e.A * e.A * e.X;
  S.D0 = (e.sg * e.A) * e.A * e.A - e.sg * (e.A * e.B * e.B);
  S.BB = e.B * e.B;
  S.AABY = e.A * e.A * e.B * e.Y;
  return S;
}

// One pass of newton_iteration's loop (cylinder.h:594-614): the condition -- at most 100
// steps while |R'(v)| >= 1e-7, R' being distance_derivative (:516-547),
//   -2 * (X - v) - 2 * B * v * (B / A * s -+ Y) / (A * s)
// -- and, when it holds, the step single_newton_iteration (:551-590),
//   v <- ((+-A A A X -+ A v v X) s + B v v v Y) / ((+-A A A -+ A B B -+ A v v +- B B v v / A) s
//         + A A B Y),
// then the nudge of a value that lands on |v| == a (the cylinder's a in every branch, as the
// reference).  The derivative and the step take the same s = sqrt(|v^2 - A^2|), computed once.
// Returns false when the loop ends (v is then final).
BZR_HD bool ellipse_search_step(const EllipseSearch &S, double a, double &v, int &steps) {
  const EllipseBranch &e = S.e;
  const double s = root_gap(v, e.A);
  const double d = -2 * (e.X - v) - S.B2 * v * (S.BA * s - e.tg * e.Y) / (e.A * s);
  if (!((fabs(d) >= 1e-7) && (steps < 100))) return false;
  const double num = (S.A3X - e.sg * (e.A * v * v * e.X)) * s + e.B * v * v * v * e.Y;
  const double den = (S.D0 - e.sg * (e.A * v * v) + e.sg * (S.BB * v * v / e.A)) * s + S.AABY;
  v = num / den;
  ++steps;
  if (fabs(v) == a) v += kDblEps;
  return true;
}

// The sector test of find_minimum_distance_to_ellipse (cylinder.h:622-673) as branch
// parameters.
BZR_HD EllipseBranch ellipse_branch(double a, double b, double xq, double yq) {
  if (((xq >= 0) && (yq >= (b / a) * xq)) || ((xq <= 0) && (yq >= (-b / a) * xq)))
    return {a, b, xq, yq, 1.0, 1.0};    // upper half, over x
  if (((xq >= 0) && (yq <= (-b / a) * xq)) || ((xq <= 0) && (yq <= (b / a) * xq)))
    return {a, b, xq, yq, -1.0, -1.0};  // lower half, over x
  if ((xq >= 0) && (yq <= (b / a) * xq) && (yq >= (-b / a) * xq))
    return {b, a, yq, xq, 1.0, -1.0};   // right sector, over y
  return {b, a, yq, xq, -1.0, 1.0};     // left sector, over y
}

// find_minimum_distance_to_ellipse after its search: the other coordinate
// +-(B / A) sqrt(A^2 - v^2) and the distance from the point.
BZR_HD double ellipse_finish(const EllipseBranch &e, double v) {
  const double s = sqrt(e.A * e.A - v * v);
  const double w = (e.sg * e.B) / e.A * s;
  return sqrt((e.X - v) * (e.X - v) + (e.Y - w) * (e.Y - w));
}

// find_minimum_distance_to_ellipse: the start at +-0.95 A, the search, the finish.
BZR_HD double ellipse_distance(double a, double b, double xq, double yq) {
  const EllipseSearch S = ellipse_search(ellipse_branch(a, b, xq, yq));
  const double percentage = 0.95;
  double v = S.e.X > 0 ? percentage * S.e.A : -percentage * S.e.A;
  int steps = 0;
  while (ellipse_search_step(S, a, v, steps)) {
  }
  return ellipse_finish(S.e, v);
}

// cylinder.h:677-759 split around its ellipse search, so that a kernel can run the searches
// of many points in lockstep: cylinder_setup takes every decision before the search (and
// returns the result when no search is needed), cylinder_finish combines the shell distance
// with the caps as the reference's region does.
struct CylinderQuery {
  EllipseSearch S;
  double a = 0.0;       // the cylinder's semi_axis_a (the search's nudge compares with it)
  double v = 0.0;       // the search's value (start: +-0.95 A)
  double top = 0.0, bottom = 0.0;
  int region = 0;       // 0 result ready; 1 inside; 2 beside the shell; 3 outside above/below
  int steps = 0;        // search steps taken
  double result = 0.0;
};

BZR_HD CylinderQuery cylinder_setup(D3 c, double a, double b, double height, const double *R,
                                    D3 p) {
  CylinderQuery q;
  const D3 lp = to_local(R, c, p);
  const double dist_top = fabs(lp.z - height / 2);
  const double dist_bottom = fabs(lp.z + height / 2);
  const double x_q = lp.x, y_q = lp.y, z_q = lp.z;
  q.top = dist_top;
  q.bottom = dist_bottom;
  q.a = a;
  if (x_q == 0 && y_q == 0) {  // isZero(point_xy)
    if ((z_q > height / 2) || (z_q < -height / 2))
      q.result = min_first(dist_top, dist_bottom);
    else
      q.result = min_first(min_first(min_first(a, b), dist_top), dist_bottom);
    return q;
  }
  const double ellipse = (x_q * x_q) / (a * a) + (y_q * y_q) / (b * b) - 1;
  if (fabs(ellipse) < kDblEps) {
    q.result = ((z_q > height / 2) || (z_q < -height / 2)) ? min_first(dist_top, dist_bottom)
                                                          : 0.0;
    return q;
  }
  if (ellipse < 0) {
    if (z_q >= height / 2) {
      q.result = dist_top;
      return q;
    }
    if (z_q <= -height / 2) {
      q.result = dist_bottom;
      return q;
    }
    q.region = 1;
  } else if (ellipse > 0) {
    q.region = ((z_q < height / 2) && (z_q > -height / 2)) ? 2 : 3;
  } else {
    q.result = -1.0;  // a NaN ellipse value (degenerate semi-axes)
    return q;
  }
  q.S = ellipse_search(ellipse_branch(a, b, x_q, y_q));
  const double percentage = 0.95;
  q.v = q.S.e.X > 0 ? percentage * q.S.e.A : -percentage * q.S.e.A;
  return q;
}

BZR_HD double cylinder_finish(const CylinderQuery &q, double v) {
  const double dist_shell = ellipse_finish(q.S.e, v);
  if (q.region == 1) return min_first(min_first(dist_shell, q.bottom), q.top);
  if (q.region == 2) return dist_shell;
  const double dist1 = sqrt(dist_shell * dist_shell + q.top * q.top);
  const double dist2 = sqrt(dist_shell * dist_shell + q.bottom * q.bottom);
  return min_first(dist1, dist2);
}

// One pass of the search's loop for a query in its search: false when it has ended.
BZR_HD bool cylinder_search_step(CylinderQuery &q) {
  return ellipse_search_step(q.S, q.a, q.v, q.steps);
}

// cylinder.h:677-759
BZR_HD double cylinder_distance(D3 c, double a, double b, double height, const double *R,
                                D3 p) {
  CylinderQuery q = cylinder_setup(c, a, b, height, R, p);
  if (q.region == 0) return q.result;
  while (cylinder_search_step(q)) {
  }
  return cylinder_finish(q, q.v);
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

// The float at or below x (the stack keeps box distances as floats: a key that is not larger
// than the distance only lets the search visit more, never less).
BZR_HD float float_below(double x) {
#if defined(__CUDA_ARCH__)
  return __double2float_rd(x);
#else
  float f = static_cast<float>(x);
  if (static_cast<double>(f) > x) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
  return f;
#endif
}

// The smallest (distance, kind, id) wins, so the order in which kinds and primitives are
// searched does not change the result.
BZR_HD void nearest_offer(NearestState &st, int kind, uint32_t geom, uint32_t id, double d) {
  if (d < st.best || (d == st.best && st.prim != 0xFFFFFFFFu &&
                      (kind < st.kind || (kind == st.kind && id < st.prim)))) {
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
                        uint32_t *stack_ref, float *stack_key, uint32_t cap) {
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
        stack_key[sp] = float_below(first1 ? d0 : d1);
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

// Search order: the smaller of the two BVH kinds first (a cheap early bound prunes the larger
// one), then the other, then cylinders (whose skip test uses the bound) and planes.
BZR_HD NearestState nearest_surface(const SceneView &S, D3 p, uint32_t *stack_ref,
                                    float *stack_key, uint32_t cap) {
  NearestState st;
  st.best = BZR_INF;
  const double ps = fmax(fmax(fabs(p.x), fabs(p.y)), fabs(p.z));
  const bool spheres_first = S.k[kSpheres].n_prims < S.k[kMesh].n_prims;
  const int order[kNumKinds] = {spheres_first ? kSpheres : kMesh,
                                spheres_first ? kMesh : kSpheres, kCylinders, kPlanes};
  for (int j = 0; j < kNumKinds; ++j) {
    const int kind = order[j];
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
