/* CPU oracle: plain-C restatement of blazeRT's closest-hit path (see bzr_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY -- the checker, never the thing measured or shipped.
 *
 * Compile with -ffp-contract=off: every expression below is written in the evaluation order of
 * the reference source it cites, with blaze's vector operations in the order fixed by
 * oracle/shim/blaze/Math.h (dot = (x0*y0 + x1*y1) + x2*y2, normalize = v * (1/|v|), ...).
 * Citations are paths inside the reference project. */
#include "bzr_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORA_NONE 0xFFFFFFFFu

/* ---------------------------------------------------------------- vector helpers (shim order) */
typedef struct {
  double e[3];
} v3;

static inline v3 mk(double a, double b, double c) {
  v3 r = {{a, b, c}};
  return r;
}
static inline v3 ld(const double *p) { return mk(p[0], p[1], p[2]); }
static inline v3 add(v3 a, v3 b) { return mk(a.e[0] + b.e[0], a.e[1] + b.e[1], a.e[2] + b.e[2]); }
static inline v3 sub(v3 a, v3 b) { return mk(a.e[0] - b.e[0], a.e[1] - b.e[1], a.e[2] - b.e[2]); }
static inline v3 mul_vs(v3 a, double s) { return mk(a.e[0] * s, a.e[1] * s, a.e[2] * s); }
static inline v3 mul_sv(double s, v3 a) { return mk(s * a.e[0], s * a.e[1], s * a.e[2]); }
static inline v3 div_vs(v3 a, double s) { return mk(a.e[0] / s, a.e[1] / s, a.e[2] / s); }
static inline double dot(v3 a, v3 b) { return (a.e[0] * b.e[0] + a.e[1] * b.e[1]) + a.e[2] * b.e[2]; }
static inline v3 cross(v3 a, v3 b) {
  return mk(a.e[1] * b.e[2] - a.e[2] * b.e[1], a.e[2] * b.e[0] - a.e[0] * b.e[2],
            a.e[0] * b.e[1] - a.e[1] * b.e[0]);
}
static inline double norm(v3 a) { return sqrt(dot(a, a)); }
static inline v3 normalize(v3 a) {
  const double len = norm(a);
  const double il = (len != 0.0) ? 1.0 / len : 0.0;
  return mul_vs(a, il);
}
/* R * v, R row-major 3x3 */
static inline v3 matvec(const double *R, v3 v) {
  return mk((R[0] * v.e[0] + R[1] * v.e[1]) + R[2] * v.e[2],
            (R[3] * v.e[0] + R[4] * v.e[1]) + R[5] * v.e[2],
            (R[6] * v.e[0] + R[7] * v.e[1]) + R[8] * v.e[2]);
}
/* trans(R) * v */
static inline v3 mattvec(const double *R, v3 v) {
  return mk((R[0] * v.e[0] + R[3] * v.e[1]) + R[6] * v.e[2],
            (R[1] * v.e[0] + R[4] * v.e[1]) + R[7] * v.e[2],
            (R[2] * v.e[0] + R[5] * v.e[1]) + R[8] * v.e[2]);
}
/* std::min(a, b) / std::max(a, b) exactly: the first argument wins ties and NaN tests. */
static inline double std_min(double a, double b) { return (b < a) ? b : a; }
static inline double std_max(double a, double b) { return (a < b) ? b : a; }
/* blazert/datatypes.h:79-85 */
static inline double product_sign(double x, double y) {
  uint64_t bx, by;
  memcpy(&bx, &x, 8);
  memcpy(&by, &y, 8);
  bx ^= (by & UINT64_C(0x8000000000000000));
  double r;
  memcpy(&r, &bx, 8);
  return r;
}
/* blazert/datatypes.h:87-93 (unity): accumulate a box into (mn, mx). */
static inline void unity(double *mn, double *mx, const double *bmin, const double *bmax) {
  for (int k = 0; k < 3; k++) {
    mn[k] = std_min(bmin[k], mn[k]);
    mx[k] = std_max(bmax[k], mx[k]);
  }
}

/* ---------------------------------------------------------------- scene */
typedef struct {
  double mn[3], mx[3];
  uint32_t leaf, axis, child[2], prim_off, prim_cnt;
} ora_node;

typedef struct {
  int present;
  uint32_t geom_id;
  long n;
  double *bmin, *bmax, *center; /* per primitive, n x 3 */
  ora_node *nodes;
  long n_nodes, cap_nodes;
  uint32_t *leaf_prims; /* primitive ids in leaf order */
  long n_leaf_prims;
  uint32_t max_depth_seen;
} ora_kind;

struct ora_scene {
  ora_kind k[4];
  long n_verts;
  double *verts, *vert_n;
  uint32_t *faces;
  double *sph_c, *sph_r;
  double *pl_c, *pl_dx, *pl_dy, *pl_rot;
  double *cy_c, *cy_a, *cy_b, *cy_h, *cy_rot;
  unsigned min_leaf, max_depth, bins;
};

static double *dup(const double *p, long n) {
  double *r = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  if (n > 0) memcpy(r, p, sizeof(double) * (size_t)n);
  return r;
}

static void alloc_kind(ora_kind *k, long n) {
  k->n = n;
  k->bmin = (double *)calloc((size_t)(3 * n + 1), sizeof(double));
  k->bmax = (double *)calloc((size_t)(3 * n + 1), sizeof(double));
  k->center = (double *)calloc((size_t)(3 * n + 1), sizeof(double));
}

/* blazert/primitives/trimesh.h:78-95, :109-130 */
static void precompute_mesh(ora_scene *s, long n_faces) {
  ora_kind *k = &s->k[0];
  alloc_kind(k, n_faces);
  s->vert_n = (double *)calloc((size_t)(3 * s->n_verts + 1), sizeof(double));
  for (long f = 0; f < n_faces; f++) {
    const uint32_t *F = s->faces + 3 * f;
    const v3 v0 = ld(s->verts + 3 * F[0]), v1 = ld(s->verts + 3 * F[1]),
             v2 = ld(s->verts + 3 * F[2]);
    /* :122-124  (v0 + v1 + v2) / 3 */
    const v3 c = div_vs(add(add(v0, v1), v2), 3.0);
    memcpy(k->center + 3 * f, c.e, 24);
    /* :109-120 */
    double mn[3], mx[3];
    memcpy(mn, v0.e, 24);
    memcpy(mx, v0.e, 24);
    unity(mn, mx, v1.e, v1.e);
    unity(mn, mx, v2.e, v2.e);
    memcpy(k->bmin + 3 * f, mn, 24);
    memcpy(k->bmax + 3 * f, mx, 24);
    /* :126-130  normalize(cross(v1 - v0, v2 - v0)) */
    const v3 e2 = sub(v2, v0), e1 = sub(v1, v0);
    const v3 fn = normalize(cross(e1, e2));
    /* :91-93  vertex_normals[v] += face_normal / 3 */
    const v3 add3 = div_vs(fn, 3.0);
    for (int j = 0; j < 3; j++) {
      double *vn = s->vert_n + 3 * F[j];
      for (int q = 0; q < 3; q++) vn[q] = vn[q] + add3.e[q];
    }
  }
}

/* blazert/primitives/sphere.h:93-100 */
static void precompute_spheres(ora_scene *s, long n) {
  ora_kind *k = &s->k[1];
  alloc_kind(k, n);
  for (long i = 0; i < n; i++) {
    for (int q = 0; q < 3; q++) {
      k->bmin[3 * i + q] = s->sph_c[3 * i + q] - s->sph_r[i];
      k->bmax[3 * i + q] = s->sph_c[3 * i + q] + s->sph_r[i];
      k->center[3 * i + q] = s->sph_c[3 * i + q];
    }
  }
}

/* std::min / std::max over an initializer list of six values (min_element / max_element). */
static void list_minmax6(const v3 *p, double *mn, double *mx) {
  for (int q = 0; q < 3; q++) {
    double a = p[0].e[q], b = p[0].e[q];
    for (int j = 1; j < 6; j++) {
      if (p[j].e[q] < a) a = p[j].e[q];
      if (b < p[j].e[q]) b = p[j].e[q];
    }
    mn[q] = a;
    mx[q] = b;
  }
}

/* blazert/primitives/plane.h:113-150 */
static void precompute_planes(ora_scene *s, long n) {
  ora_kind *k = &s->k[2];
  alloc_kind(k, n);
  const double th = DBL_MIN; /* plane.h:82 thickness */
  for (long i = 0; i < n; i++) {
    const v3 c = ld(s->pl_c + 3 * i);
    const double dx = s->pl_dx[i], dy = s->pl_dy[i];
    const double *R = s->pl_rot + 9 * i;
    v3 p[6];
    p[0] = add(c, matvec(R, mk(-dx / 2.0, -dy / 2.0, 0.0)));
    p[1] = add(c, matvec(R, mk(dx / 2.0, -dy / 2.0, 0.0)));
    p[2] = add(c, matvec(R, mk(-dx / 2.0, dy / 2.0, 0.0)));
    p[3] = add(c, matvec(R, mk(dx / 2.0, dy / 2.0, 0.0)));
    p[4] = add(c, matvec(R, mk(0.0, 0.0, -th)));
    p[5] = add(c, matvec(R, mk(0.0, 0.0, th)));
    list_minmax6(p, k->bmin + 3 * i, k->bmax + 3 * i);
    memcpy(k->center + 3 * i, c.e, 24);
  }
}

/* blazert/primitives/cylinder.h:115-147 */
static void precompute_cylinders(ora_scene *s, long n) {
  ora_kind *k = &s->k[3];
  alloc_kind(k, n);
  for (long i = 0; i < n; i++) {
    const v3 c = ld(s->cy_c + 3 * i);
    const double a = s->cy_a[i], b = s->cy_b[i], h = s->cy_h[i];
    const double *R = s->cy_rot + 9 * i;
    const v3 ra = matvec(R, mk(a, 0.0, 0.0)), rb = matvec(R, mk(0.0, b, 0.0)),
             rh = matvec(R, mk(0.0, 0.0, h / 2.0));
    v3 p[6];
    p[0] = add(c, ra); /* a1 */
    p[1] = add(c, rb); /* b1 */
    p[2] = sub(c, ra); /* a2 */
    p[3] = sub(c, rb); /* b2 */
    p[4] = add(c, rh); /* h1 */
    p[5] = sub(c, rh); /* h2 */
    list_minmax6(p, k->bmin + 3 * i, k->bmax + 3 * i);
    memcpy(k->center + 3 * i, c.e, 24);
  }
}

/* ---------------------------------------------------------------- binned SAH builder */
typedef struct {
  double mn[3], mx[3];
  uint32_t count;
  double cost;
} ora_bin;

typedef struct {
  ora_kind *k;
  uint32_t *idx;
  ora_bin *bins;
  unsigned min_leaf, max_depth, nbins;
} build_ctx;

static void bin_reset(ora_bin *b) {
  for (int q = 0; q < 3; q++) {
    b->mn[q] = DBL_MAX;
    b->mx[q] = -DBL_MAX;
  }
  b->count = 0;
  b->cost = 0.0;
}

/* blazert/bvh/binbuffer.h:16-19 */
static double box_surface(const double *mn, const double *mx) {
  const double b0 = fabs(mx[0] - mn[0]), b1 = fabs(mx[1] - mn[1]), b2 = fabs(mx[2] - mn[2]);
  return 2.0 * ((b0 * b1 + b1 * b2) + b2 * b0);
}

/* blazert/bvh/binbuffer.h:66-95 (sort_collection_into_bins) and :114-167
 * (find_best_split_binned).  Returns the cut axis; cut_pos receives the per-axis cut. */
static unsigned best_split(build_ctx *c, long begin, long end, const double *mn, const double *mx,
                           double *cut_pos) {
  const unsigned nb = c->nbins;
  ora_bin *bins = c->bins;
  for (unsigned i = 0; i < 3 * nb; i++) bin_reset(&bins[i]);
  double inv_size[3];
  for (int q = 0; q < 3; q++) {
    const double size = mx[q] - mn[q];
    inv_size[q] = (size > 0.0) ? 1.0 / size : 0.0;
  }
  for (long it = begin; it < end; it++) {
    const uint32_t p = c->idx[it];
    const double *bmn = c->k->bmin + 3 * p, *bmx = c->k->bmax + 3 * p;
    const double *ctr = c->k->center + 3 * p;
    for (int j = 0; j < 3; j++) {
      /* (center - min) * inv_size * (bins - 1) */
      const double nc = ((ctr[j] - mn[j]) * inv_size[j]) * (double)(nb - 1);
      /* min(bins-1, unsigned(max(0u, unsigned(round(nc))))): the double->unsigned conversion
       * behaves as on x86-64 (through a 64-bit signed integer). */
      uint32_t id = (uint32_t)(int64_t)round(nc);
      if (id > nb - 1) id = nb - 1;
      ora_bin *b = &bins[j * nb + id];
      b->count++;
      unity(b->mn, b->mx, bmn, bmx);
    }
  }
  double min_cost[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
  for (int j = 0; j < 3; j++) {
    uint64_t count = 0;
    double amn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, amx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (unsigned i = nb - 1; i > 0; i--) {
      ora_bin *b = &bins[j * nb + i];
      unity(amn, amx, b->mn, b->mx);
      count += b->count;
      b->cost = (double)count * box_surface(amn, amx);
    }
    count = 0;
    for (int q = 0; q < 3; q++) {
      amn[q] = DBL_MAX;
      amx[q] = -DBL_MAX;
    }
    unsigned min_bin = 1;
    for (unsigned i = 0; i < nb - 1; i++) {
      ora_bin *b = &bins[j * nb + i];
      const ora_bin *nx = &bins[j * nb + i + 1];
      unity(amn, amx, b->mn, b->mx);
      count += b->count;
      const double cost = (double)count * box_surface(amn, amx) + nx->cost;
      if (cost < min_cost[j]) {
        min_cost[j] = cost;
        min_bin = i + 1;
      }
    }
    cut_pos[j] = (double)min_bin * ((mx[j] - mn[j]) / (double)nb) + mn[j];
  }
  unsigned axis = 0;
  if (min_cost[0] > min_cost[1]) axis = 1;
  if (min_cost[axis] > min_cost[2]) axis = 2;
  return axis;
}

/* std::partition for bidirectional iterators (two cursors moving inward, swapping
 * misplaced pairs), as libstdc++ implements it; the leaf primitive order depends on it. */
static long partition_range(build_ctx *c, long first, long last, unsigned axis, double cut) {
  const double *ctr = c->k->center;
  for (;;) {
    for (;;) {
      if (first == last) return first;
      if (ctr[3 * c->idx[first] + axis] < cut)
        ++first;
      else
        break;
    }
    --last;
    for (;;) {
      if (first == last) return first;
      if (!(ctr[3 * c->idx[last] + axis] < cut))
        --last;
      else
        break;
    }
    const uint32_t tmp = c->idx[first];
    c->idx[first] = c->idx[last];
    c->idx[last] = tmp;
    ++first;
  }
}

static long push_node(ora_kind *k) {
  if (k->n_nodes == k->cap_nodes) {
    k->cap_nodes = k->cap_nodes ? 2 * k->cap_nodes : 64;
    k->nodes = (ora_node *)realloc(k->nodes, sizeof(ora_node) * (size_t)k->cap_nodes);
  }
  ora_node *nd = &k->nodes[k->n_nodes];
  memset(nd, 0, sizeof(*nd));
  nd->leaf = ORA_NONE;
  nd->axis = ORA_NONE;
  nd->child[0] = nd->child[1] = ORA_NONE;
  return k->n_nodes++;
}

/* blazert/bvh/builder.h:84-115 (build_recursive), :133-148 (create_leaf), :167-183
 * (create_branch), :201-226 (split) */
static uint32_t build_rec(build_ctx *c, long begin, long end, unsigned depth) {
  ora_kind *k = c->k;
  const long off = push_node(k);
  if (k->max_depth_seen < depth) k->max_depth_seen = depth;
  const unsigned n = (unsigned)(end - begin);
  double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (long it = begin; it < end; it++) {  /* blazert/bvh/bbox.h:27-39 */
    const uint32_t p = c->idx[it];
    unity(mn, mx, k->bmin + 3 * p, k->bmax + 3 * p);
  }
  ora_node *nd = &k->nodes[off];
  memcpy(nd->mn, mn, 24);
  memcpy(nd->mx, mx, 24);
  if (n <= c->min_leaf || depth >= c->max_depth) {
    nd->leaf = 1;
    nd->prim_off = (uint32_t)k->n_leaf_prims;
    nd->prim_cnt = n;
    for (long it = begin; it < end; it++) k->leaf_prims[k->n_leaf_prims++] = c->idx[it];
    return (uint32_t)off;
  }
  double cut_pos[3];
  unsigned cut_axis = best_split(c, begin, end, mn, mx, cut_pos);
  long mid = begin;
  for (unsigned axis_try = 0; axis_try < 3; axis_try++) {
    mid = partition_range(c, begin, end, cut_axis, cut_pos[cut_axis]);
    if (mid == begin || mid == end) {
      mid = begin + ((end - begin) >> 1);
      cut_axis = (cut_axis + 1) % 3;
    } else {
      break;
    }
  }
  nd->leaf = 0;
  nd->axis = cut_axis;
  const uint32_t c0 = build_rec(c, begin, mid, depth + 1);
  k->nodes[off].child[0] = c0;
  const uint32_t c1 = build_rec(c, mid, end, depth + 1);
  k->nodes[off].child[1] = c1;
  return (uint32_t)off;
}

/* blazert/bvh/builder.h:46-65 */
static void build_kind(ora_scene *s, ora_kind *k) {
  build_ctx c;
  c.k = k;
  c.min_leaf = s->min_leaf;
  c.max_depth = s->max_depth;
  c.nbins = s->bins;
  c.idx = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(k->n + 1));
  for (long i = 0; i < k->n; i++) c.idx[i] = (uint32_t)i;
  c.bins = (ora_bin *)malloc(sizeof(ora_bin) * 3 * (size_t)s->bins);
  k->leaf_prims = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(k->n + 1));
  k->n_leaf_prims = 0;
  k->max_depth_seen = 0;
  build_rec(&c, 0, k->n, 0);
  free(c.idx);
  free(c.bins);
}

ora_scene *ora_scene_create(const int *order, int n_order, const double *verts, long n_verts,
                            const uint32_t *faces, long n_faces, const double *sph_c,
                            const double *sph_r, long n_sph, const double *pl_c,
                            const double *pl_dx, const double *pl_dy, const double *pl_rot,
                            long n_pl, const double *cy_c, const double *cy_a, const double *cy_b,
                            const double *cy_h, const double *cy_rot, long n_cy, unsigned min_leaf,
                            unsigned max_depth, unsigned bins, uint32_t *geom_ids) {
  ora_scene *s = (ora_scene *)calloc(1, sizeof(ora_scene));
  s->min_leaf = min_leaf;
  s->max_depth = max_depth;
  s->bins = bins;
  uint32_t next_id = 0;
  for (int j = 0; j < n_order; j++) {
    const int kind = order[j];
    uint32_t id = ORA_NONE;
    if (kind >= 0 && kind < 4 && !s->k[kind].present) { /* blazert/scene.h:227-346 */
      s->k[kind].present = 1;
      id = s->k[kind].geom_id = next_id++;
      switch (kind) {
        case 0:
          s->n_verts = n_verts;
          s->verts = dup(verts, 3 * n_verts);
          s->faces = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(3 * n_faces + 1));
          if (n_faces) memcpy(s->faces, faces, sizeof(uint32_t) * 3 * (size_t)n_faces);
          precompute_mesh(s, n_faces);
          break;
        case 1:
          s->sph_c = dup(sph_c, 3 * n_sph);
          s->sph_r = dup(sph_r, n_sph);
          precompute_spheres(s, n_sph);
          break;
        case 2:
          s->pl_c = dup(pl_c, 3 * n_pl);
          s->pl_dx = dup(pl_dx, n_pl);
          s->pl_dy = dup(pl_dy, n_pl);
          s->pl_rot = dup(pl_rot, 9 * n_pl);
          precompute_planes(s, n_pl);
          break;
        case 3:
          s->cy_c = dup(cy_c, 3 * n_cy);
          s->cy_a = dup(cy_a, n_cy);
          s->cy_b = dup(cy_b, n_cy);
          s->cy_h = dup(cy_h, n_cy);
          s->cy_rot = dup(cy_rot, 9 * n_cy);
          precompute_cylinders(s, n_cy);
          break;
      }
    }
    if (geom_ids) geom_ids[j] = id;
  }
  /* blazert/scene.h:91-115 (commit) */
  for (int kind = 0; kind < 4; kind++)
    if (s->k[kind].present) build_kind(s, &s->k[kind]);
  return s;
}

void ora_scene_destroy(ora_scene *s) {
  if (!s) return;
  for (int i = 0; i < 4; i++) {
    free(s->k[i].bmin);
    free(s->k[i].bmax);
    free(s->k[i].center);
    free(s->k[i].nodes);
    free(s->k[i].leaf_prims);
  }
  free(s->verts);
  free(s->vert_n);
  free(s->faces);
  free(s->sph_c);
  free(s->sph_r);
  free(s->pl_c);
  free(s->pl_dx);
  free(s->pl_dy);
  free(s->pl_rot);
  free(s->cy_c);
  free(s->cy_a);
  free(s->cy_b);
  free(s->cy_h);
  free(s->cy_rot);
  free(s);
}

long ora_scene_tree(const ora_scene *s, int kind, double *bmin, double *bmax, uint32_t *leaf,
                    uint32_t *axis, uint32_t *children, uint32_t *prim_off, uint32_t *prim_cnt,
                    uint32_t *prim_ids, long prim_cap) {
  if (kind < 0 || kind > 3 || !s->k[kind].present) return -1;
  const ora_kind *k = &s->k[kind];
  if (!bmin) return k->n_nodes;
  uint32_t running = 0; /* leaves are created in node order, so offsets run in node order */
  for (long i = 0; i < k->n_nodes; i++) {
    const ora_node *nd = &k->nodes[i];
    memcpy(bmin + 3 * i, nd->mn, 24);
    memcpy(bmax + 3 * i, nd->mx, 24);
    leaf[i] = nd->leaf;
    axis[i] = nd->axis;
    children[2 * i] = nd->child[0];
    children[2 * i + 1] = nd->child[1];
    prim_off[i] = running;
    prim_cnt[i] = nd->leaf == 1 ? nd->prim_cnt : 0;
    running += prim_cnt[i];
  }
  for (long i = 0; i < k->n_leaf_prims && i < prim_cap; i++) prim_ids[i] = k->leaf_prims[i];
  return k->n_nodes;
}

/* ---------------------------------------------------------------- ray and traversal */
typedef struct {
  v3 org, dir, inv;
  unsigned sign[3];
  double tmin, tmax;
  int any_hit; /* Ray::AnyHit::yes (blazert/ray.h:24-34) */
} ora_ray;

/* blazert/ray.h:56-65: direction normalized, inverse and sign from the RAW direction. */
static ora_ray make_ray(const double *o, const double *d, double tmin, double tmax) {
  ora_ray r;
  r.org = ld(o);
  const v3 raw = ld(d);
  r.dir = normalize(raw);
  r.inv = mk(1.0 / raw.e[0], 1.0 / raw.e[1], 1.0 / raw.e[2]);
  for (int i = 0; i < 3; i++) r.sign[i] = raw.e[i] < 0.0 ? 1u : 0u;
  r.tmin = tmin;
  r.tmax = tmax;
  r.any_hit = 0;
  return r;
}

/* blazert/bvh/intersect.h:33-51 */
static int node_test(double *min_d, double *max_d, const double *bmn, const double *bmx,
                     const ora_ray *r) {
  const double l1 = 1.0 + 4.0 * DBL_EPSILON;
  for (int i = 0; i < 3; i++) {
    double lo = r->sign[i] ? bmx[i] : bmn[i];
    double hi = r->sign[i] ? bmn[i] : bmx[i];
    lo = (lo - r->org.e[i]) * r->inv.e[i];
    hi = ((hi - r->org.e[i]) * r->inv.e[i]) * l1;
    *min_d = std_max(lo, *min_d);
    *max_d = std_min(hi, *max_d);
  }
  return *min_d <= *max_d;
}

/* Intersector state (TriangleIntersector / SphereIntersector / PlaneIntersector /
 * CylinderIntersector) after prepare_traversal. */
typedef struct {
  double tmin, hit;
  double uv[2];
  uint32_t prim;
  v3 normal; /* planes and cylinders compute it inside intersect_primitive */
} ora_isect;

static void prepare(ora_isect *st, const ora_ray *r) {
  st->tmin = r->tmin;
  st->hit = r->tmax;
  st->uv[0] = st->uv[1] = 0.0;
  st->prim = ORA_NONE;
  st->normal = mk(0.0, 0.0, 0.0);
}

/* blazert/primitives/trimesh.h:153-181, with the Triangle of :19-43 (a = v0, b = v2 - v0,
 * c = v0 - v1). */
static int isect_triangle(const ora_scene *s, ora_isect *st, uint32_t prim, const ora_ray *r) {
  const double tolerance = 4.0 * DBL_EPSILON;
  const uint32_t *F = s->faces + 3 * prim;
  const v3 a = ld(s->verts + 3 * F[0]), vb = ld(s->verts + 3 * F[1]), vc = ld(s->verts + 3 * F[2]);
  const v3 e2 = sub(vc, a); /* tri.b */
  const v3 e1 = sub(a, vb); /* tri.c */
  const v3 c = sub(a, r->org);
  const v3 rr = cross(r->dir, c);
  const double det = dot(cross(e1, e2), r->dir);
  const double abs_det = fabs(det);
  const double u = product_sign(dot(rr, e2), det);
  const double v = product_sign(dot(rr, e1), det);
  const double w = (abs_det - u) - v;
  if (u >= -tolerance && v >= -tolerance && w >= -tolerance) {
    const double t = product_sign(dot(cross(e1, e2), c), det);
    if (t >= abs_det * st->tmin && abs_det * st->hit > t) {
      const double inv_det = 1.0 / abs_det;
      st->hit = t * inv_det;
      st->uv[0] = u * inv_det;
      st->uv[1] = v * inv_det;
      st->prim = prim;
      return 1;
    }
  }
  return 0;
}

/* blazert/primitives/sphere.h:135-177 */
static int isect_sphere(const ora_scene *s, ora_isect *st, uint32_t prim, const ora_ray *r) {
  const v3 org = r->org, dir = r->dir;
  const v3 center = ld(s->sph_c + 3 * prim);
  const double radius = s->sph_r[prim];
  const v3 v = sub(org, center);
  const double A = dot(dir, dir);
  const double B = 2.0 * dot(v, dir);
  const double C = dot(v, v) - radius * radius;
  const double D = B * B - (4.0 * A) * C;
  if (D < 0.0) return 0;
  const double Q = sqrt(D);
  const double rcpA = 1.0 / A;
  const double t0 = (0.5 * rcpA) * (-B - Q);
  const double t1 = (0.5 * rcpA) * (-B + Q);
  if ((t0 > st->tmin) && (t0 < st->hit)) {
    st->hit = norm(mul_sv(t0, dir));
    st->prim = prim;
    return 1;
  }
  if ((t1 > st->tmin) && (t1 < st->hit)) {
    st->hit = norm(mul_sv(t1, dir));
    st->prim = prim;
    return 1;
  }
  return 0;
}

/* blazert/primitives/plane.h:180-270 */
static int isect_plane(const ora_scene *s, ora_isect *st, uint32_t prim, const ora_ray *r) {
  const v3 center = ld(s->pl_c + 3 * prim);
  const double dx = s->pl_dx[prim], dy = s->pl_dy[prim];
  const double *R = s->pl_rot + 9 * prim;
  const v3 org = mattvec(R, sub(r->org, center));
  const v3 dir = mattvec(R, r->dir);
  const double t1 = -org.e[2] / dir.e[2];
  const v3 ic = add(org, mul_sv(t1, dir));
  const double tnear = st->tmin, tfar = st->hit;
  const double x_min = -dx / 2, x_max = dx / 2, y_min = -dy / 2, y_max = dy / 2;
  const int in_t = (t1 > tnear) && (t1 < tfar);
  if (!in_t) return 0;
  const double x = ic.e[0], y = ic.e[1];
  const double sz = org.e[2] / fabs(org.e[2]);
  v3 n;
  if ((x > x_min) && (x < x_max) && (y > y_min) && (y < y_max)) {
    n = mul_sv(sz, matvec(R, mk(0.0, 0.0, 1.0)));
  } else if ((x == x_min) && (x < x_max) && (y > y_min) && (y < y_max)) { /* edges */
    n = matvec(R, mk(-1.0, 0.0, sz));
  } else if ((x > x_min) && (x == x_max) && (y > y_min) && (y < y_max)) {
    n = matvec(R, mk(1.0, 0.0, sz));
  } else if ((x > x_min) && (x < x_max) && (y == y_min) && (y < y_max)) {
    n = matvec(R, mk(0.0, -1.0, sz));
  } else if ((x > x_min) && (x < x_max) && (y > y_min) && (y == y_max)) {
    n = matvec(R, mk(0.0, 1.0, sz));
  } else if ((x == x_min) && (x < x_max) && (y == y_min) && (y < y_max)) { /* corners */
    n = matvec(R, mk(-1.0, -1.0, sz));
  } else if ((x == x_min) && (x < x_max) && (y > y_min) && (y == y_max)) {
    n = matvec(R, mk(-1.0, 1.0, sz));
  } else if ((x > x_min) && (x == x_max) && (y == y_min) && (y < y_max)) {
    n = matvec(R, mk(1.0, -1.0, sz));
  } else if ((x > x_min) && (x == x_max) && (y > y_min) && (y == y_max)) {
    n = matvec(R, mk(1.0, 1.0, sz));
  } else {
    return 0;
  }
  st->normal = n;
  st->hit = norm(mul_sv(t1, dir));
  st->prim = prim;
  return 1;
}

/* (R * n) / norm(n) -- the "Ng" of cylinder.h */
static v3 cyl_ng(const double *R, v3 n) { return div_vs(matvec(R, n), norm(n)); }

static int cyl_hit(ora_isect *st, uint32_t prim, v3 normal, double t, v3 dir) {
  st->normal = normal;
  st->hit = norm(mul_sv(t, dir));
  st->prim = prim;
  return 1;
}

/* blazert/primitives/cylinder.h:181-495.  No closest-hit or t-range test: a later cylinder
 * overwrites an earlier hit. */
static int isect_cylinder(const ora_scene *s, ora_isect *st, uint32_t prim, const ora_ray *r) {
  const v3 center = ld(s->cy_c + 3 * prim);
  const double a = s->cy_a[prim], b = s->cy_b[prim], h = s->cy_h[prim];
  const double *R = s->cy_rot + 9 * prim;
  const v3 org = mattvec(R, sub(r->org, center));
  const v3 dir = mattvec(R, r->dir);
  const double x0 = org.e[0], y0 = org.e[1], z0 = org.e[2];
  const double j = dir.e[0], k = dir.e[1], l = dir.e[2];
  const double h2 = h / 2.0, mh2 = -h / 2.0;
  /* the quadratic of the elliptic shell, written as in the reference */
#define CYL_ABC()                                                                         \
  const double A = a * a * k * k + b * b * j * j;                                         \
  const double B = a * a * k * y0 + b * b * j * x0;                                       \
  const double C = a * a * k * k + b * b * j * j - j * j * y0 * y0 + 2 * j * k * x0 * y0 - \
                   k * k * x0 * x0;
#define CYL_T01()                                               \
  const double t0 = 1.0 / A * (-B + a * b * sqrt(C));           \
  const double t1 = -1.0 / A * (B + a * b * sqrt(C));           \
  const v3 i0 = add(org, mul_vs(dir, t0));                      \
  const v3 i1 = add(org, mul_vs(dir, t1));
#define SHELL_N(ic) mk(2 * (ic).e[0] / (a * a), 2 * (ic).e[1] / (b * b), 0.0)

  if (z0 > h2) { /* area 1 */
    if (l == 0) return 0;
    const double tc = (h2 - z0) / l;
    if (tc < 0) return 0;
    const v3 ic = add(org, mul_sv(tc, dir));
    if (b * b * ic.e[0] * ic.e[0] + a * a * ic.e[1] * ic.e[1] <= a * a * b * b) {
      return cyl_hit(st, prim, cyl_ng(R, mk(0.0, 0.0, 1.0)), tc, dir);
    } else {
      CYL_ABC();
      if (C < 0) return 0;
      CYL_T01();
      if ((t1 > 0) && (t1 < t0) && (i1.e[2] <= h2) && (i1.e[2] >= mh2))
        return cyl_hit(st, prim, cyl_ng(R, SHELL_N(i1)), t1, dir);
      if ((t0 > 0) && (t0 < t1) && (i0.e[2] <= h2) && (i0.e[2] >= mh2))
        return cyl_hit(st, prim, cyl_ng(R, SHELL_N(i0)), t0, dir);
    }
  } else if (z0 < mh2) { /* area 2 */
    if (l == 0) return 0;
    const double tc = (mh2 - z0) / l;
    if (tc < 0) return 0;
    const v3 ic = add(org, mul_sv(tc, dir));
    if (b * b * ic.e[0] * ic.e[0] + a * a * ic.e[1] * ic.e[1] <= a * a * b * b) {
      return cyl_hit(st, prim, cyl_ng(R, mk(0.0, 0.0, -1.0)), tc, dir);
    } else {
      CYL_ABC();
      if (C < 0) return 0;
      CYL_T01();
      if ((t1 > 0) && (t1 < t0) && (i1.e[2] <= h2) && (i1.e[2] >= mh2))
        return cyl_hit(st, prim, cyl_ng(R, SHELL_N(i1)), t1, dir);
      if ((t0 > 0) && (t0 < t1) && (i0.e[2] <= h2) && (i0.e[2] >= mh2))
        return cyl_hit(st, prim, cyl_ng(R, SHELL_N(i0)), t0, dir);
    }
  } else if ((z0 > mh2) && (z0 < h2) && (x0 * x0 * b * b + y0 * y0 * a * a > a * a * b * b)) {
    /* area 3 */
    CYL_ABC();
    if (C < 0) return 0;
    CYL_T01();
    if ((t1 > 0) && (t1 < t0) && (i1.e[2] <= h2) && (i1.e[2] >= mh2))
      return cyl_hit(st, prim, cyl_ng(R, SHELL_N(i1)), t1, dir);
    if ((t0 > 0) && (t0 < t1) && (i0.e[2] <= h2) && (i0.e[2] >= mh2))
      return cyl_hit(st, prim, cyl_ng(R, SHELL_N(i0)), t0, dir);
  }
  /* area 4 */
  if ((z0 >= mh2) && (z0 <= h2) && (x0 * x0 * b * b + y0 * y0 * a * a <= a * a * b * b)) {
    if (l == 0) {
      if ((z0 == mh2) || (z0 == h2)) return 0;
      CYL_ABC();
      if (C < 0) return 0;
      CYL_T01();
      if ((t1 > 0) && (i1.e[2] <= h2) && (i1.e[2] >= mh2))
        return cyl_hit(st, prim, cyl_ng(R, SHELL_N(i1)), t1, dir);
      if ((t0 > 0) && (i0.e[2] <= h2) && (i0.e[2] >= mh2))
        return cyl_hit(st, prim, cyl_ng(R, SHELL_N(i0)), t0, dir);
    } else if ((j == 0.0) && (k == 0)) {
      if (b * b * x0 * x0 + a * a * y0 * y0 == a * a * b * b) return 0;
      if (l < 0) {
        const double tc = (mh2 - z0) / l;
        return cyl_hit(st, prim, cyl_ng(R, mk(0.0, 0.0, -1.0)), tc, dir);
      }
      if (l > 0) {
        const double tc = (h2 - z0) / l;
        return cyl_hit(st, prim, cyl_ng(R, mk(0.0, 0.0, 1.0)), tc, dir);
      }
    } else {
      CYL_ABC();
      if (C < 0) return 0;
      CYL_T01();
      if ((t1 > 0) && (i1.e[2] <= h2) && (i1.e[2] >= mh2))
        return cyl_hit(st, prim, cyl_ng(R, SHELL_N(i1)), t1, dir);
      if ((t0 > 0) && (i0.e[2] <= h2) && (i0.e[2] >= mh2)) /* unrotated normal, :462-463 */
        return cyl_hit(st, prim, SHELL_N(i0), t0, dir);
      if (l < 0) {
        const double tc = (mh2 - z0) / l;
        return cyl_hit(st, prim, cyl_ng(R, mk(0.0, 0.0, -1.0)), tc, dir);
      }
      if (l > 0) {
        const double tc = (h2 - z0) / l;
        return cyl_hit(st, prim, cyl_ng(R, mk(0.0, 0.0, 1.0)), tc, dir);
      }
    }
  }
#undef CYL_ABC
#undef CYL_T01
#undef SHELL_N
  return 0;
}

static int isect_prim(const ora_scene *s, int kind, ora_isect *st, uint32_t prim,
                      const ora_ray *r) {
  switch (kind) {
    case 0: return isect_triangle(s, st, prim, r);
    case 1: return isect_sphere(s, st, prim, r);
    case 2: return isect_plane(s, st, prim, r);
    default: return isect_cylinder(s, st, prim, r);
  }
}

/* post_traversal: trimesh.h:133-143, sphere.h:107-114, plane.h:153-159, cylinder.h:154-160 */
static v3 post_normal(const ora_scene *s, int kind, const ora_isect *st, const ora_ray *r) {
  switch (kind) {
    case 0: {
      const uint32_t *F = s->faces + 3 * st->prim;
      const double u = st->uv[0], v = st->uv[1];
      const double w = (1.0 - u) - v;
      const v3 n0 = ld(s->vert_n + 3 * F[0]), n1 = ld(s->vert_n + 3 * F[1]),
               n2 = ld(s->vert_n + 3 * F[2]);
      return normalize(add(add(mul_sv(w, n0), mul_sv(u, n1)), mul_sv(v, n2)));
    }
    case 1: {
      const v3 c = ld(s->sph_c + 3 * st->prim);
      return normalize(sub(add(r->org, mul_sv(st->hit, r->dir)), c));
    }
    default:
      return normalize(st->normal);
  }
}

typedef struct {
  double t, uv[2];
  v3 normal;
  uint32_t prim;
} ora_hit;

/* blazert/bvh/accel.h:80-120 (traverse) with intersect_leaf (intersect.h:67-78). */
static int traverse_kind(const ora_scene *s, int kind, const ora_ray *r, ora_hit *out,
                         uint32_t *cnt_nodes, uint32_t *cnt_prims, uint32_t *peak) {
  const ora_kind *k = &s->k[kind];
  uint32_t stack[256];
  unsigned ss = 0;
  stack[ss++] = 0;
  ora_isect st;
  prepare(&st, r);
  double hit_distance = r->tmax;
  while (ss > 0) {
    double max_d = hit_distance, min_d = r->tmin;
    const ora_node *nd = &k->nodes[stack[ss - 1]];
    ss--;
    if (cnt_nodes) (*cnt_nodes)++;
    if (node_test(&min_d, &max_d, nd->mn, nd->mx, r)) {
      if (nd->leaf != 1) {
        const unsigned near = r->sign[nd->axis];
        if (ss + 2 > 256) break; /* deeper than any tree built with max_depth < 254 */
        stack[ss++] = nd->child[1 - near];
        stack[ss++] = nd->child[near];
        if (peak && ss > *peak) *peak = ss;
      } else {
        /* intersect_leaf: with any_hit the leaf stops at its first hit, and the traversal
         * with it (intersect.h:73-75, accel.h:109-110) */
        int hit = 0;
        for (uint32_t q = 0; q < nd->prim_cnt; q++) {
          if (cnt_prims) (*cnt_prims)++;
          hit += isect_prim(s, kind, &st, k->leaf_prims[nd->prim_off + q], r);
          if (hit && r->any_hit) break;
        }
        if (hit) {
          hit_distance = st.hit;
          if (r->any_hit) break;
        }
      }
    }
  }
  const int hit = st.hit < r->tmax;
  if (hit) {
    out->t = st.hit;
    out->uv[0] = st.uv[0];
    out->uv[1] = st.uv[1];
    out->prim = st.prim;
    out->normal = post_normal(s, kind, &st, r);
  }
  return hit;
}

/* blazert/scene.h:161-210 (intersect1): kinds in the fixed order triangles, spheres, planes,
 * cylinders; the first copies unconditionally, later ones only when strictly closer. */
static int intersect1(const ora_scene *s, const ora_ray *r, ora_hit *rh, uint32_t *geom,
                      uint32_t *counters, uint32_t *peak) {
  int hit = 0;
  ora_hit tmp;
  for (int kind = 0; kind < 4; kind++) {
    if (!s->k[kind].present) continue;
    const int h = traverse_kind(s, kind, r, &tmp, counters ? counters + kind : NULL,
                                counters ? counters + 4 + kind : NULL, peak);
    if (h && (kind == 0 || tmp.t < rh->t)) {
      *rh = tmp;
      *geom = s->k[kind].geom_id;
      hit = 1;
    }
  }
  return hit;
}

void ora_scene_intersect(const ora_scene *s, long n, const double *org, const double *dir,
                         const double *tmin, const double *tmax, double *t, double *uv,
                         double *normal, uint32_t *prim, uint32_t *geom, uint8_t *hit,
                         uint32_t *counters, uint32_t *stack_peak, int nthreads) {
  ora_scene_intersect_ex(s, n, org, dir, tmin, tmax, 0, t, uv, normal, prim, geom, hit, counters,
                         stack_peak, nthreads);
}

void ora_scene_intersect_ex(const ora_scene *s, long n, const double *org, const double *dir,
                            const double *tmin, const double *tmax, int any_hit, double *t,
                            double *uv, double *normal, uint32_t *prim, uint32_t *geom,
                            uint8_t *hit, uint32_t *counters, uint32_t *stack_peak,
                            int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
#else
  (void)nthreads;
#endif
  for (long i = 0; i < n; i++) {
    ora_ray r = make_ray(org + 3 * i, dir + 3 * i, tmin ? tmin[i] : 0.0,
                         tmax ? tmax[i] : DBL_MAX);
    r.any_hit = any_hit != 0;
    ora_hit rh;
    rh.t = DBL_MAX; /* RayHit defaults, blazert/ray.h:80-84 */
    rh.uv[0] = rh.uv[1] = 0.0;
    rh.normal = mk(0.0, 0.0, 0.0);
    rh.prim = ORA_NONE;
    uint32_t g = ORA_NONE, peak = 1;
    uint32_t *cnt = counters ? counters + 8 * i : NULL;
    if (cnt) memset(cnt, 0, 8 * sizeof(uint32_t));
    const int h = intersect1(s, &r, &rh, &g, cnt, &peak);
    if (t) t[i] = rh.t;
    if (uv) {
      uv[2 * i] = rh.uv[0];
      uv[2 * i + 1] = rh.uv[1];
    }
    if (normal) memcpy(normal + 3 * i, rh.normal.e, 24);
    if (prim) prim[i] = rh.prim;
    if (geom) geom[i] = g;
    if (hit) hit[i] = (uint8_t)h;
    if (stack_peak) stack_peak[i] = peak;
  }
}

int ora_intersect_node(double *min_distance, double *max_distance, const double bmin[3],
                       const double bmax[3], const double org[3], const double raw_dir[3]) {
  const ora_ray r = make_ray(org, raw_dir, 0.0, DBL_MAX);
  return node_test(min_distance, max_distance, bmin, bmax, &r);
}

int ora_intersect_primitive0(const ora_scene *s, int kind, const double org[3],
                             const double raw_dir[3], double tmin, double tmax, double *t,
                             double *uv, double *normal, uint32_t *prim) {
  const ora_ray r = make_ray(org, raw_dir, tmin, tmax);
  ora_isect st;
  prepare(&st, &r);
  const int h = isect_prim(s, kind, &st, 0, &r);
  if (h) {
    const v3 n = post_normal(s, kind, &st, &r);
    *t = st.hit;
    uv[0] = st.uv[0];
    uv[1] = st.uv[1];
    memcpy(normal, n.e, 24);
    *prim = st.prim;
  } else {
    *t = DBL_MAX;
    uv[0] = uv[1] = 0.0;
    normal[0] = normal[1] = normal[2] = 0.0;
    *prim = ORA_NONE;
  }
  return h;
}

int ora_traverse_kind(const ora_scene *s, int kind, const double org[3], const double raw_dir[3],
                      double tmin, double tmax, double *t, double *uv, double *normal,
                      uint32_t *prim) {
  if (kind < 0 || kind > 3 || !s->k[kind].present) return -1;
  const ora_ray r = make_ray(org, raw_dir, tmin, tmax);
  ora_hit rh;
  rh.t = DBL_MAX;
  rh.uv[0] = rh.uv[1] = 0.0;
  rh.normal = mk(0.0, 0.0, 0.0);
  rh.prim = ORA_NONE;
  const int h = traverse_kind(s, kind, &r, &rh, NULL, NULL, NULL);
  *t = rh.t;
  uv[0] = rh.uv[0];
  uv[1] = rh.uv[1];
  memcpy(normal, rh.normal.e, 24);
  *prim = rh.prim;
  return h;
}

/* ------------------------------------------------------------------------------------------
 * Distance to surface (blazert/primitives/sphere.h:179-182, plane.h:272-284,
 * cylinder.h:498-759; triangles through trimesh_distance.h:37-218). */

/* cylinder.h:508-513 */
static double ellipse_equation(double a, double b, double x, double y) {
  return (x * x) / (a * a) + (y * y) / (b * b) - 1;
}

/* the conditional square root every branch of cylinder.h:516-590 starts with */
static double gap_sqrt(double val, double s) {
  return (val * val > s * s) ? sqrt(val * val - s * s) : sqrt(s * s - val * val);
}

/* branch: 0 upper/x, 1 lower/x, 2 upper/y, 3 lower/y (cylinder.h:516-547) */
static double distance_derivative(int branch, double a, double b, double xq, double yq,
                                  double val) {
  switch (branch) {
    case 0: {
      const double sq = gap_sqrt(val, a);
      return -2 * (xq - val) - 2 * b * val * (b / a * sq - yq) / (a * sq);
    }
    case 1: {
      const double sq = gap_sqrt(val, a);
      return -2 * (xq - val) - 2 * b * val * (b / a * sq + yq) / (a * sq);
    }
    case 2: {
      const double sq = gap_sqrt(val, b);
      return -2 * (yq - val) - 2 * a * val * (a / b * sq + xq) / (b * sq);
    }
    default: {
      const double sq = gap_sqrt(val, b);
      return -2 * (yq - val) - 2 * a * val * (a / b * sq - xq) / (b * sq);
    }
  }
}

/* cylinder.h:551-590 */
static double single_newton_iteration(int branch, double a, double b, double xq, double yq,
                                      double val) {
  switch (branch) {
    case 0: {
      const double sq = gap_sqrt(val, a);
      return ((a * a * a * xq - a * val * val * xq) * sq + b * val * val * val * yq) /
             ((a * a * a - a * b * b - a * val * val + b * b * val * val / a) * sq + a * a * b * yq);
    }
    case 1: {
      const double sq = gap_sqrt(val, a);
      return ((-a * a * a * xq + a * val * val * xq) * sq + b * val * val * val * yq) /
             ((-a * a * a + a * b * b + a * val * val - b * b * val * val / a) * sq + a * a * b * yq);
    }
    case 2: {
      const double sq = gap_sqrt(val, b);
      return ((b * b * b * yq - b * val * val * yq) * sq + a * val * val * val * xq) /
             ((b * b * b - b * a * a - b * val * val + a * a * val * val / b) * sq + b * b * a * xq);
    }
    default: {
      const double sq = gap_sqrt(val, b);
      return ((-b * b * b * yq + b * val * val * yq) * sq + a * val * val * val * xq) /
             ((-b * b * b + b * a * a + b * val * val - a * a * val * val / b) * sq + b * b * a * xq);
    }
  }
}

/* cylinder.h:594-614: epsilon 1e-7 for double, at most 100 iterations */
static double newton_iteration(int branch, double a, double b, double xq, double yq, double x0) {
  double val0 = x0, cnt = 0;
  while ((fabs(distance_derivative(branch, a, b, xq, yq, val0)) >= 1e-7) && (cnt < 100)) {
    const double val = single_newton_iteration(branch, a, b, xq, yq, val0);
    val0 = val;
    cnt++;
    if (fabs(val0) == a) val0 += DBL_EPSILON;
  }
  return val0;
}

/* cylinder.h:622-673 (the distance of the returned pair) */
static double min_distance_to_ellipse(double a, double b, double xq, double yq) {
  const double percentage = 0.95;
  if (((xq >= 0) && (yq >= (b / a) * xq)) || ((xq <= 0) && (yq >= (-b / a) * xq))) {
    const double x0 = xq > 0 ? percentage * a : -percentage * a;
    const double x_min = newton_iteration(0, a, b, xq, yq, x0);
    const double sq = sqrt(a * a - x_min * x_min);
    const double y_min = b / a * sq;
    return sqrt((xq - x_min) * (xq - x_min) + (yq - y_min) * (yq - y_min));
  }
  if (((xq >= 0) && (yq <= (-b / a) * xq)) || ((xq <= 0) && (yq <= (b / a) * xq))) {
    const double x0 = xq > 0 ? percentage * a : -percentage * a;
    const double x_min = newton_iteration(1, a, b, xq, yq, x0);
    const double sq = sqrt(a * a - x_min * x_min);
    const double y_min = -b / a * sq;
    return sqrt((xq - x_min) * (xq - x_min) + (yq - y_min) * (yq - y_min));
  }
  if ((xq >= 0) && (yq <= (b / a) * xq) && (yq >= (-b / a) * xq)) {
    const double y0 = yq > 0 ? percentage * b : -percentage * b;
    const double y_min = newton_iteration(2, a, b, xq, yq, y0);
    const double sq = sqrt(b * b - y_min * y_min);
    const double x_min = a / b * sq;
    return sqrt((yq - y_min) * (yq - y_min) + (xq - x_min) * (xq - x_min));
  }
  {
    const double y0 = yq > 0 ? percentage * b : -percentage * b;
    const double y_min = newton_iteration(3, a, b, xq, yq, y0);
    const double sq = sqrt(b * b - y_min * y_min);
    const double x_min = -a / b * sq;
    return sqrt((yq - y_min) * (yq - y_min) + (xq - x_min) * (xq - x_min));
  }
}

/* cylinder.h:677-759 */
static double cylinder_distance(const ora_scene *s, uint32_t id, v3 p) {
  const double *R = s->cy_rot + 9 * id;
  const v3 lp = mattvec(R, sub(p, ld(s->cy_c + 3 * id)));
  const double h = s->cy_h[id];
  const double dist_top = fabs(lp.e[2] - h / 2);
  const double dist_bottom = fabs(lp.e[2] + h / 2);
  const double x_q = lp.e[0], y_q = lp.e[1], z_q = lp.e[2];
  const double a = s->cy_a[id], b = s->cy_b[id];
  if (x_q == 0 && y_q == 0) {
    if ((z_q > h / 2) || (z_q < -h / 2)) return std_min(dist_top, dist_bottom);
    return std_min(std_min(std_min(a, b), dist_top), dist_bottom);
  }
  const double ellipse = ellipse_equation(a, b, x_q, y_q);
  if (fabs(ellipse) < DBL_EPSILON) {
    if ((z_q > h / 2) || (z_q < -h / 2)) return std_min(dist_top, dist_bottom);
    return 0.0;
  }
  if (ellipse < 0) {
    if (z_q >= h / 2) return dist_top;
    if (z_q <= -h / 2) return dist_bottom;
    return std_min(std_min(min_distance_to_ellipse(a, b, x_q, y_q), dist_bottom), dist_top);
  }
  if (ellipse > 0) {
    const double shell = min_distance_to_ellipse(a, b, x_q, y_q);
    if ((z_q < h / 2) && (z_q > -h / 2)) return shell;
    return std_min(sqrt(shell * shell + dist_top * dist_top),
                   sqrt(shell * shell + dist_bottom * dist_bottom));
  }
  return -1;
}

/* trimesh_distance.h:177-218 with r0..r6 (:37-163) */
static v3 closest_point_on_triangle(v3 v0, v3 v1, v3 v2, v3 p) {
  const v3 E0 = sub(v1, v0), E1 = sub(v2, v0), D = sub(v0, p);
  const double a = dot(E0, E0), b = dot(E0, E1), c = dot(E1, E1);
  const double d = dot(E0, D), e = dot(E1, D);
  const double det = a * c - b * b;
  double sv = b * e - c * d, tv = b * d - a * e;
  if (sv + tv <= det) {
    if (sv < 0) {
      if (tv < 0) { /* r4 */
        if (d < 0) {
          tv = 0;
          sv = (-d >= a) ? 1 : -d / a;
        } else {
          sv = 0;
          tv = (e >= 0) ? 0 : ((-e >= c) ? 1 : -e / c);
        }
      } else { /* r3 */
        sv = 0;
        tv = (e >= 0) ? 0 : ((-e >= c) ? 1 : -e / c);
      }
    } else if (tv < 0) { /* r5 */
      tv = 0;
      sv = (d >= 0) ? 0 : ((-d >= a) ? 1 : -d / a);
    } else { /* r0 */
      const double inv_det = 1.0 / det;
      sv *= inv_det;
      tv *= inv_det;
    }
  } else if (sv < 0) { /* r2 */
    const double tmp0 = b + d, tmp1 = c + e;
    if (tmp1 > tmp0) {
      const double numer = tmp1 - tmp0, denom = a - 2.0 * b + c;
      sv = (numer >= denom) ? 1 : numer / denom;
      tv = 1.0 - sv;
    } else {
      sv = 0;
      tv = (tmp1 <= 0) ? 1 : ((e >= 0) ? 0 : -e / c);
    }
  } else if (tv < 0) { /* r6 */
    const double tmp0 = b + e, tmp1 = a + d;
    if (tmp1 > tmp0) {
      const double numer = tmp1 - tmp0, denom = a - 2.0 * b + c;
      tv = (numer >= denom) ? 1 : numer / denom;
      sv = 1.0 - tv;
    } else {
      tv = 0;
      sv = (tmp1 <= 0) ? 1 : ((d >= 0) ? 0 : -d / a);
    }
  } else { /* r1 */
    const double numer = c + e - b - d;
    if (numer <= 0) {
      sv = 0;
    } else {
      const double denom = a - 2.0 * b + c;
      sv = (numer >= denom) ? 1 : numer / denom;
    }
    tv = 1.0 - sv;
  }
  return add(add(v0, mul_sv(sv, E0)), mul_sv(tv, E1));
}

double ora_distance_one(const ora_scene *s, int kind, uint32_t id, const double point[3],
                        double closest[3]) {
  const v3 p = ld(point);
  switch (kind) {
    case 0: {
      const uint32_t *F = s->faces + 3 * id;
      const v3 c = closest_point_on_triangle(ld(s->verts + 3 * F[0]), ld(s->verts + 3 * F[1]),
                                             ld(s->verts + 3 * F[2]), p);
      if (closest) memcpy(closest, c.e, 24);
      return norm(sub(c, p));
    }
    case 1: /* sphere.h:179-182 */
      return fabs(norm(sub(ld(s->sph_c + 3 * id), p)) - s->sph_r[id]);
    case 2: { /* plane.h:272-284 */
      const v3 c = ld(s->pl_c + 3 * id);
      const v3 lp = mattvec(s->pl_rot + 9 * id, sub(p, c));
      const double dx = s->pl_dx[id] / 2, dy = s->pl_dy[id] / 2;
      if ((lp.e[0] >= c.e[0] - dx) && (lp.e[0] <= c.e[0] + dx) && (lp.e[1] >= c.e[1] - dy) &&
          (lp.e[1] <= c.e[1] + dy))
        return fabs(lp.e[2]);
      return DBL_MAX;
    }
    default:
      return cylinder_distance(s, id, p);
  }
}

void ora_distance_to_surface(const ora_scene *s, int kind, long n, const uint32_t *ids,
                             const double *points, double *distance, double *closest) {
  for (long i = 0; i < n; i++)
    distance[i] = ora_distance_one(s, kind, ids[i], points + 3 * i,
                                   closest ? closest + 3 * i : NULL);
}

/* The scene-level nearest surface by exhaustion: kinds in the order triangles, spheres, planes,
 * cylinders, primitives by increasing id, the first strictly smaller distance kept. */
void ora_closest_surface(const ora_scene *s, long n, const double *points, double *distance,
                         uint32_t *prim, uint32_t *geom) {
  for (long i = 0; i < n; i++) {
    double best = INFINITY;
    uint32_t bp = 0xFFFFFFFFu, bg = 0xFFFFFFFFu;
    for (int kind = 0; kind < 4; kind++) {
      if (!s->k[kind].present) continue;
      for (long id = 0; id < s->k[kind].n; id++) {
        const double d = ora_distance_one(s, kind, (uint32_t)id, points + 3 * i, NULL);
        if (d < best) {
          best = d;
          bp = (uint32_t)id;
          bg = s->k[kind].geom_id;
        }
      }
    }
    distance[i] = best;
    if (prim) prim[i] = bp;
    if (geom) geom[i] = bg;
  }
}
