/* CPU oracle for the blazeRT closest-hit ray query: a plain-C restatement of the reference's
 * algorithm (binned-SAH build, stack traversal, the four intersectors, intersect1's merge).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it, and only as the checker; the product (libblazert_b200.so) never calls it.
 *
 * Parity status: pinned.  The restatement is checked bit-for-bit against the reference's own
 * code compiled here (oracle/ref_driver.cpp -> oracle/_ref/) on every committed golden fixture
 * (tests/golden/), and against the reference test suite's known-answer vectors.
 *
 * Array conventions: vec3 arrays are n x 3 row-major doubles, rotation matrices n x 9 row-major.
 * Kinds: 0 triangle mesh, 1 spheres, 2 planes, 3 cylinders. */
#ifndef BZR_ORACLE_H_
#define BZR_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_scene ora_scene;

ora_scene *ora_scene_create(const int *order, int n_order, const double *verts, long n_verts,
                            const uint32_t *faces, long n_faces, const double *sph_c,
                            const double *sph_r, long n_sph, const double *pl_c,
                            const double *pl_dx, const double *pl_dy, const double *pl_rot,
                            long n_pl, const double *cy_c, const double *cy_a, const double *cy_b,
                            const double *cy_h, const double *cy_rot, long n_cy, unsigned min_leaf,
                            unsigned max_depth, unsigned bins, uint32_t *geom_ids);
void ora_scene_destroy(ora_scene *s);

/* intersect1 over n rays; counters (n x 8 uint32 or NULL) receive per kind the number of nodes
 * popped and tested (slots 0-3) and of primitive tests (slots 4-7).  stack_peak (n or NULL)
 * receives the largest traversal-stack occupancy the ray reached. */
void ora_scene_intersect(const ora_scene *s, long n, const double *org, const double *dir,
                         const double *tmin, const double *tmax, double *t, double *uv,
                         double *normal, uint32_t *prim, uint32_t *geom, uint8_t *hit,
                         uint32_t *counters, uint32_t *stack_peak, int nthreads);

/* ora_scene_intersect with every ray's any_hit flag set to `any_hit` (Ray::AnyHit::yes,
 * blazert/ray.h:24-34): each kind's traversal stops at the first leaf hit it accepts. */
void ora_scene_intersect_ex(const ora_scene *s, long n, const double *org, const double *dir,
                            const double *tmin, const double *tmax, int any_hit, double *t,
                            double *uv, double *normal, uint32_t *prim, uint32_t *geom,
                            uint8_t *hit, uint32_t *counters, uint32_t *stack_peak,
                            int nthreads);

/* Node dump with the same layout as oracle/ref_driver.cpp's ref_scene_tree. */
long ora_scene_tree(const ora_scene *s, int kind, double *bmin, double *bmax, uint32_t *leaf,
                    uint32_t *axis, uint32_t *children, uint32_t *prim_off, uint32_t *prim_cnt,
                    uint32_t *prim_ids, long prim_cap);

/* Slab test of one box (blazert/bvh/intersect.h:33-51) for unit tests of the node KATs. */
int ora_intersect_node(double *min_distance, double *max_distance, const double bmin[3],
                       const double bmax[3], const double org[3], const double raw_dir[3]);

/* Primitive tests against primitive 0 of a one-kind collection, without a BVH
 * (test/test_primitives/assert_helper.h:123-139 pattern).  Returns hit; writes t, uv[2],
 * normal[3], prim. */
int ora_intersect_primitive0(const ora_scene *s, int kind, const double org[3],
                             const double raw_dir[3], double tmin, double tmax, double *t,
                             double *uv, double *normal, uint32_t *prim);

/* Per-kind traversal without the intersect1 merge (blazert/bvh/accel.h:60-120). */
int ora_traverse_kind(const ora_scene *s, int kind, const double org[3], const double raw_dir[3],
                      double tmin, double tmax, double *t, double *uv, double *normal,
                      uint32_t *prim);

/* distance_to_surface of primitive ids[i] of one kind for n points (blazert/primitives/
 * sphere.h:179-182, plane.h:272-284, cylinder.h:677-759); triangles: closest_point_on_triangle
 * (trimesh_distance.h:177-218) on the face's vertices, distance norm(closest - p), closest
 * (n x 3 or NULL) receives the points. */
void ora_distance_to_surface(const ora_scene *s, int kind, long n, const uint32_t *ids,
                             const double *points, double *distance, double *closest);
double ora_distance_one(const ora_scene *s, int kind, uint32_t id, const double point[3],
                        double closest[3]);

/* Nearest surface over the whole scene by exhaustion: kinds in the order triangles, spheres,
 * planes, cylinders, primitives by increasing id, the first strictly smaller distance kept
 * (+inf and 0xFFFFFFFF when none). */
void ora_closest_surface(const ora_scene *s, long n, const double *points, double *distance,
                         uint32_t *prim, uint32_t *geom);

#ifdef __cplusplus
}
#endif
#endif
