/* blazert_b200 -- B200-native closest-hit ray queries behind blazeRT's Scene API.
 *
 * C-ABI of libblazert_b200.so.  Plain pointers and sizes only.  Every function returns an
 * int status (BZR_OK == 0, negative on error); bzr_last_error_string() describes the last
 * failure of the calling thread.
 *
 * The entry points replace the reference's compile-time Scene interface (paths inside the
 * reference project):
 *   bzr_scene_create / _destroy   BlazertScene<T> ctor / dtor       blazert/scene.h:38-73
 *   bzr_add_mesh                  BlazertScene<T>::add_mesh         blazert/scene.h:227-240
 *   bzr_add_spheres               BlazertScene<T>::add_spheres      blazert/scene.h:258-271
 *   bzr_add_planes                BlazertScene<T>::add_planes       blazert/scene.h:293-307
 *   bzr_add_cylinders             BlazertScene<T>::add_cylinders    blazert/scene.h:331-346
 *   bzr_commit                    BlazertScene<T>::commit           blazert/scene.h:91-115
 *                                 with BVHBuildOptions              blazert/bvh/options.h:15-29
 *   bzr_intersect1                intersect1(scene, ray, rayhit)    blazert/scene.h:161-210
 *                                 with Ray / RayHit                 blazert/ray.h:56-85
 *   bzr_intersectN                new: intersect1 over a batch of rays, one GPU launch
 *   bzr_intersect1_ex / _ex       the two above with ray flags: BZR_RAY_ANY_HIT for
 *                                 Ray::AnyHit::yes              blazert/ray.h:24-65,
 *                                 blazert/bvh/intersect.h:67-78, blazert/bvh/accel.h:105-111
 *   bzr_adjoint_hit               new: gradients of the outputs (differentiation form)
 *   bzr_batch_*                   new: many scenes per launch, CUDA graph (batching form)
 *   bzr_work_counts, bzr_scene_check, bzr_scene_stats, bzr_scene_tune
 *                                 new: measurement, error reporting and tuning
 *
 * Semantics kept from the reference:
 *   - add_* may be called once per primitive kind and only before commit; otherwise the
 *     returned geom id is UINT32_MAX (the reference's static_cast<unsigned>(-1)) and the status
 *     is BZR_ESTATE.  Geom ids count up from 0 in add order.
 *   - intersect1 semantics per ray: per-kind BVHs traversed in the fixed order triangles,
 *     spheres, planes, cylinders; the first (triangles) is copied when hit, later kinds only
 *     when strictly closer.  A ray that hits nothing keeps the default RayHit: hit_distance =
 *     DBL_MAX, uv = normal = 0, prim_id = geom_id = UINT32_MAX, hit = 0.
 *   - Directions need not be unit length: as in the reference the ray direction is normalized
 *     and the slab test uses the inverse of the raw direction.
 * Deliberate difference: add_* COPY the caller's arrays (the reference keeps const& to them), so
 * the caller may free them after the call.  Results are identical.
 *
 * Array layout: vec3 arrays are n x 3 row-major float64; rotation matrices n x 9 row-major
 * float64 (R[3*i + j] = R(i, j)); faces n x 3 uint32.
 */
#ifndef BLAZERT_B200_H_
#define BLAZERT_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BZR_OK 0
#define BZR_EINVAL (-1)       /* bad argument (null pointer, size, mode) */
#define BZR_ESTATE (-2)       /* wrong scene state (add after commit, second add, not committed) */
#define BZR_ENOMEM (-3)       /* host or device allocation failed */
#define BZR_ECUDA (-4)        /* a CUDA runtime call failed */
#define BZR_ETIMEOUT (-5)     /* a bounded wait for the device ran out */
#define BZR_EDEVICE_FLAG (-6) /* a kernel's own bounds check fired (error word set) */
#define BZR_ENODEV (-7)       /* no CUDA device */

#define BZR_INVALID_ID 0xFFFFFFFFu

/* Precision of the traversal (the primitive tests and the closest-hit compare are always FP64). */
#define BZR_MODE_FP64 0  /* slab tests in FP64: bit-exact with the reference */
#define BZR_MODE_MIXED 1 /* conservative FP32 slab tests, exact FP64 re-test at leaves */

typedef struct bzr_scene bzr_scene;

/* BVHBuildOptions (blazert/bvh/options.h:15-29); defaults 4 / 28 / 64. */
typedef struct {
  uint32_t min_leaf_primitives; /* a node with this many primitives or fewer becomes a leaf */
  uint32_t max_tree_depth;
  uint32_t bin_size;
} bzr_build_options;

/* RayHit (blazert/ray.h:72-85). */
typedef struct {
  double normal[3];
  double uv[2];
  double hit_distance;
  uint32_t prim_id;
  uint32_t geom_id;
} bzr_rayhit;

int bzr_scene_create(bzr_scene **out);
int bzr_scene_destroy(bzr_scene *scene);

int bzr_add_mesh(bzr_scene *scene, const double *vertices, size_t n_vertices,
                 const uint32_t *faces, size_t n_faces, uint32_t *geom_id);
int bzr_add_spheres(bzr_scene *scene, const double *centers, const double *radii, size_t n,
                    uint32_t *geom_id);
int bzr_add_planes(bzr_scene *scene, const double *centers, const double *dxs, const double *dys,
                   const double *rotations, size_t n, uint32_t *geom_id);
int bzr_add_cylinders(bzr_scene *scene, const double *centers, const double *semi_axes_a,
                      const double *semi_axes_b, const double *heights, const double *rotations,
                      size_t n, uint32_t *geom_id);

/* Builds the per-kind binned-SAH BVHs (the reference's tree, node for node; on the device for
 * kinds of at least 65,536 primitives, see bzr_commit_ex), flattens them into the device
 * layout and uploads them to the current CUDA device.  options may be NULL for the
 * defaults. */
int bzr_commit(bzr_scene *scene, const bzr_build_options *options);

/* bzr_commit with flags (the device builder has no counterpart in the reference; the tree it
 * builds is the reference's).  The device build gives each kind's BVH from the same binned
 * SAH with the same bins and leaf size, node for node (node boxes can differ only in the sign
 * of a zero bound), when every box and centre is finite, min_leaf_primitives >= 1 and
 * bin_size <= 256; otherwise, or if it fails, the host builds.  By default (flags 0, and in
 * bzr_commit) kinds of at least 65,536 primitives are built on the device;
 * BZR_COMMIT_GPU_BUILD asks for the device at every size, BZR_COMMIT_HOST_BUILD for the host
 * at every size. */
#define BZR_COMMIT_GPU_BUILD 1u
#define BZR_COMMIT_HOST_BUILD 2u
int bzr_commit_ex(bzr_scene *scene, const bzr_build_options *options, uint32_t flags);

/* One ray (Ray{origin, direction, tmin, tmax}); *hit receives intersect1's return value. */
int bzr_intersect1(const bzr_scene *scene, const double origin[3], const double direction[3],
                   double tmin, double tmax, bzr_rayhit *rayhit, int *hit);

/* Ray flags (the reference's per-ray enums, blazert/ray.h:24-34).  BZR_RAY_ANY_HIT is
 * Ray::AnyHit::yes: in each kind's traversal the first primitive hit a leaf accepts ends the
 * leaf and the traversal (blazert/bvh/intersect.h:73-75, blazert/bvh/accel.h:109-110); the
 * kinds are still merged as intersect1 does.  Used for shadow rays, where only hit / miss
 * matters (the reported hit need not be the closest).  CullBackFace has no flag: the reference
 * does not implement it (blazert/ray.h:52). */
#define BZR_RAY_ANY_HIT 1u

/* bzr_intersect1 with ray flags (0 or BZR_RAY_ANY_HIT). */
int bzr_intersect1_ex(const bzr_scene *scene, const double origin[3], const double direction[3],
                      double tmin, double tmax, uint32_t ray_flags, bzr_rayhit *rayhit,
                      int *hit);

/* A batch of n rays, structure-of-arrays.  Inputs: origins, directions (n x 3); tmin, tmax (n,
 * or NULL for 0 and DBL_MAX).  Outputs (each may be NULL to skip it): hit_distance (n), uv
 * (n x 2), normal (n x 3), prim_id, geom_id (n), hit (n, 0/1).
 * Either ALL given arrays are host memory -- copied to and from the device inside the call,
 * which returns when the results are in place -- or ALL are device memory of the scene's
 * device, in which case the work is queued on `stream` (a cudaStream_t, NULL for the default
 * stream) and the call returns without waiting.  Mixed placement is BZR_EINVAL. */
int bzr_intersectN(const bzr_scene *scene, size_t n, const double *origins,
                   const double *directions, const double *tmin, const double *tmax,
                   double *hit_distance, double *uv, double *normal, uint32_t *prim_id,
                   uint32_t *geom_id, uint8_t *hit, int mode, void *stream);

/* bzr_intersectN with ray flags applied to every ray of the batch (0 or BZR_RAY_ANY_HIT). */
int bzr_intersectN_ex(const bzr_scene *scene, size_t n, const double *origins,
                      const double *directions, const double *tmin, const double *tmax,
                      double *hit_distance, double *uv, double *normal, uint32_t *prim_id,
                      uint32_t *geom_id, uint8_t *hit, int mode, uint32_t ray_flags,
                      void *stream);

/* bzr_intersectN for callers that cannot allocate device memory while they trace (no
 * counterpart in the reference) -- for example a renderer plugin traced from its host
 * application's frame loop, where a cudaMalloc/cudaFree would synchronise the whole device, or
 * a service whose device memory budget is handed out up front.  Same arguments and results as
 * bzr_intersectN, but device arrays only, at most 1,048,576 rays per call (larger batches get
 * BZR_EINVAL), and no coherence sort.  The call allocates nothing: its scratch is one 12 MiB
 * static device array per GPU, held until the process exits.  All calls on a device share that
 * array; calls whose GPU work overlaps race -- order them on one stream.  The first call on each
 * device looks up the array's address and keeps it; make it before any stream capture, and do
 * not use this entry point on a device after a cudaDeviceReset of it in the same process. */
int bzr_intersectN_noalloc(const bzr_scene *scene, size_t n, const double *origins,
                           const double *directions, const double *tmin, const double *tmax,
                           double *hit_distance, double *uv, double *normal, uint32_t *prim_id,
                           uint32_t *geom_id, uint8_t *hit, int mode, void *stream);

/* Batching form (no counterpart in the reference): many committed scenes of one device, each
 * with its own batch of rays, traced together -- one persistent kernel per primitive kind for
 * all scenes -- with the launch sequence captured in a CUDA graph and replayed while the
 * arguments stay the same.  Results per scene equal bzr_intersectN on that scene. */
typedef struct bzr_batch bzr_batch;
int bzr_batch_create(bzr_batch **out, const bzr_scene *const *scenes, size_t n_scenes);
int bzr_batch_destroy(bzr_batch *batch);
/* Rays of scene s are [ray_offsets[s], ray_offsets[s+1]) of the concatenated device arrays
 * (ray_offsets: host array of n_scenes + 1, starting at 0).  hit_distance is required; other
 * outputs may be NULL.  scene_done_ns (device, n_scenes + 1, or NULL) receives each scene's
 * completion time and, in its last entry, the batch start time (GPU global timer, ns).
 * Queued on `stream`. */
int bzr_batch_intersect(bzr_batch *batch, const uint64_t *ray_offsets, const double *origins,
                        const double *directions, const double *tmin, const double *tmax,
                        double *hit_distance, double *uv, double *normal, uint32_t *prim_id,
                        uint32_t *geom_id, uint8_t *hit, uint64_t *scene_done_ns, int mode,
                        void *stream);
/* Waits for `stream` and reports the batch kernels' error word (as bzr_scene_check). */
int bzr_batch_check(bzr_batch *batch, void *stream, uint32_t *flags);
/* Launch shape of the batch's kernels: BZR_TUNE_BLOCK (64, 128, 256 threads per block),
 * BZR_TUNE_STACK (0 thread-local, 1 shared memory), BZR_TUNE_STACK_DEPTH (32 or 64 entries of
 * the thread-local stack), BZR_TUNE_SORT (1: each scene's rays are traced in the order of
 * their direction octant and origin Morton code in the scene's box, sorted inside the graph;
 * batches of at most 4,096 scenes) or BZR_TUNE_NODE_WIDTH (2 or 8, the mixed mode's walk);
 * see bzr_scene_tune.  Drops the cached graph; the next
 * bzr_batch_intersect captures a new one.  Results do not change. */
int bzr_batch_tune(bzr_batch *batch, int option, int64_t value);

/* Adjoint of the closest-hit outputs (no counterpart in the reference): given a batch's
 * forward results (as returned by bzr_intersectN) and upstream gradients dL/dhit_distance (n),
 * dL/duv (n x 2), dL/dnormal (n x 3) -- each may be NULL for zero -- computes dL/d(triangle
 * vertices) (n_vertices x 3), dL/d(sphere centres) (n x 3), dL/d(sphere radii), dL/d(ray
 * origins) and dL/d(raw ray directions) (n x 3 each); any output may be NULL.  The hit
 * primitive is held fixed (recomputed from prim_id, no re-traversal).  Rays whose hit is a
 * plane or cylinder get zero gradients and set kernel error bit 8 (read by bzr_scene_check).
 * Device arrays only; queued on `stream`. */
int bzr_adjoint_hit(const bzr_scene *scene, size_t n, const double *origins,
                    const double *directions, const double *hit_distance, const uint32_t *prim_id,
                    const uint32_t *geom_id, const uint8_t *hit, const double *grad_t,
                    const double *grad_uv, const double *grad_normal, double *grad_vertices,
                    double *grad_centers, double *grad_radii, double *grad_origins,
                    double *grad_directions, void *stream);

/* Work of a batch (no counterpart in the reference; a measurement aid): runs the counting
 * variant of the FP64 kernel over n rays and returns per kind (0 mesh, 1 spheres, 2 planes,
 * 3 cylinders) the number of box tests -- the reference's node pops, blazert/bvh/accel.h:94-97
 * -- in totals[0..3] and of primitive tests (blazert/bvh/intersect.h:71-76) in totals[4..7].
 * Arrays as for bzr_intersectN; returns when the totals are in place. */
int bzr_work_counts(const bzr_scene *scene, size_t n, const double *origins,
                    const double *directions, const double *tmin, const double *tmax,
                    uint64_t totals[8], void *stream);
/* The same for either mode (BZR_MODE_FP64 or BZR_MODE_MIXED), with per kind in totals[0..3]
 * the box tests (FP64: as above; mixed: the root test plus every child of every wide node
 * fetched), in totals[4..7] the primitive tests, in totals[8..11] the node fetches (FP64
 * internal nodes, or wide nodes) and in totals[12..15] the leaf fetches (FP64: leaves whose
 * primitives run; mixed: leaf records read, each with its exact FP64 box test). */
int bzr_work_counts_ex(const bzr_scene *scene, size_t n, const double *origins,
                       const double *directions, const double *tmin, const double *tmax,
                       int mode, uint64_t totals[16], void *stream);

/* Waits for the scene's queued work (bounded by timeout_ms; <= 0 waits without bound) and
 * reports the kernels' error word: BZR_OK, BZR_EDEVICE_FLAG (with *flags receiving the bits)
 * or BZR_ETIMEOUT. */
int bzr_scene_check(const bzr_scene *scene, void *stream, int timeout_ms, uint32_t *flags);

/* Tuning knobs of a committed scene (no counterpart in the reference; they change speed,
 * never results).  BZR_TUNE_SORT: 1 sorts each batch of at least BZR_TUNE_SORT_MIN_RAYS rays
 * (default 65536) by direction octant and origin Morton code before tracing, so that the rays
 * of a warp take similar paths (needs finite scene bounds); 0 (the default) traces in the
 * caller's order. */
#define BZR_TUNE_SORT 1
#define BZR_TUNE_SORT_MIN_RAYS 2
/* Launch shape of the traversal kernels: threads per block (64, 128 -- the default -- or 256);
 * traversal-stack storage (0: a thread-local array when the tree's stack fits its 64 entries,
 * the default; 1: shared memory sized from the tree); rays a warp takes from the work counter
 * per fetch (32 -- the default --, 64, 128, or 0 for exactly the lanes that are idle). */
#define BZR_TUNE_BLOCK 3
#define BZR_TUNE_STACK 4
#define BZR_TUNE_CHUNK 5
/* Host-array calls: the batch is split into at most this many chunks (1 to 32, default 8) of
 * at least BZR_TUNE_HOST_MIN_CHUNK rays (default 131,072), pipelined as copies in, kernels and
 * copies out. */
#define BZR_TUNE_HOST_CHUNKS 6
#define BZR_TUNE_HOST_MIN_CHUNK 7
/* Rays of an extra first and last chunk of host-array calls (0, the default: none), which
 * shortens the copies that do not overlap a kernel; used when the batch exceeds 4x it. */
#define BZR_TUNE_HOST_EDGE 8
/* Host-array calls: each chunk's kernels use 1/value (1 to 8, default 1) of the grid, so that
 * chunks on the pipeline's three streams can run side by side. */
#define BZR_TUNE_HOST_GRID_DIV 9
/* Top-level nodes (0 to 256, default 0) each block of the traversal kernels copies into shared
 * memory at launch and reads from there: the first nodes of the breadth-first node array the
 * kernel walks (the FP64 nodes, or the wide nodes of the mixed path), which every ray visits. */
#define BZR_TUNE_TOP_NODES 10
/* Entries of the traversal kernels' thread-local stack (batches only, bzr_batch_tune): 32 or
 * 64 (the default); 32 only when every scene's tree needs at most 32. */
#define BZR_TUNE_STACK_DEPTH 11
/* Node width of a batch's walk in BZR_MODE_MIXED (batches only, bzr_batch_tune): 8 (the
 * default) walks the 8-wide nodes with the FP32 child tests, 2 the binary FP64 nodes of the FP64
 * mode.  Both process the same leaves in the same order, so the results are the same bits;
 * BZR_MODE_FP64 always walks the binary nodes. */
#define BZR_TUNE_NODE_WIDTH 12
int bzr_scene_tune(bzr_scene *scene, int option, int64_t value);

/* Statistics of the last commit: per kind (0 mesh, 1 spheres, 2 planes, 3 cylinders) the
 * number of reference BVH nodes, the maximum depth and the host build time in seconds. */
int bzr_scene_stats(const bzr_scene *scene, int kind, uint64_t *n_nodes, uint32_t *max_depth,
                    double *build_seconds);

/* The reference's BVHBuildStatistics (blazert/bvh/statistics.h:11-38) of one kind's BVH
 * (0 triangles, 1 spheres, 2 planes, 3 cylinders) as built at commit: deepest node, leaf and
 * branch node counts, fewest and most primitives in a leaf, failed partition attempts (the
 * reference's bad_splits, builder.h:217-221) and the build time.  The reference's
 * Scene::commit drops these; here they are kept per kind. */
typedef struct bzr_build_statistics {
  uint32_t max_tree_depth;
  uint32_t leaf_nodes;
  uint32_t max_num_prims_per_leaf;
  uint32_t min_num_prims_per_leaf;
  uint32_t branch_nodes;
  uint32_t bad_splits;
  double build_seconds;
} bzr_build_statistics;
int bzr_scene_build_statistics(const bzr_scene *scene, int kind, bzr_build_statistics *out);

/* Node arrays of a committed scene's BVH of one kind (0 triangles, 1 spheres, 2 planes,
 * 3 cylinders) in the reference's DFS node order (blazert/bvh/node.h:15-41): per node its box
 * (3 + 3 doubles), leaf flag, split axis, two child indices and, for leaves, its primitive
 * count; prim_ids receives the leaves' primitives in node order (up to prim_cap).  Returns
 * the node count (call with NULL arrays to size them) or a negative status.  For tests and
 * diagnostics: compares a build against the reference's tree. */
long bzr_scene_tree(const bzr_scene *scene, int kind, double *bmin, double *bmax, uint32_t *leaf,
                    uint32_t *axis, uint32_t *children, uint32_t *prim_cnt, uint32_t *prim_ids,
                    long prim_cap);

/* Distance from points to given primitives of one kind (0 triangles, 1 spheres, 2 planes,
 * 3 cylinders): distance[i] = distance_to_surface(primitive prim_ids[i], points[3i..3i+2]),
 * bit for bit the reference's per-primitive function
 *   spheres    blazert/primitives/sphere.h:179-182    |norm(center - p) - radius|
 *   planes     blazert/primitives/plane.h:272-284     |local z| inside the rectangle test,
 *                                                     DBL_MAX outside it
 *   cylinders  blazert/primitives/cylinder.h:677-759  shell (Newton search on the ellipse), caps
 * and for triangles closest_point_on_triangle (blazert/primitives/trimesh_distance.h:177-218)
 * on the face's vertices with distance norm(closest - p); closest (n x 3, triangles only, may
 * be NULL) receives those points.  All arrays host memory (the call returns when the results
 * are written; an id outside the kind gives NaN there and the call returns BZR_EINVAL) or all
 * device memory (queued on stream; an id outside the kind gives NaN and sets the error word
 * bzr_scene_check reads). */
int bzr_distance_to_surface(const bzr_scene *scene, int kind, size_t n, const uint32_t *prim_ids,
                            const double *points, double *distance, double *closest,
                            void *stream);

/* Nearest surface of the whole scene per point: distance[i] = the smallest
 * bzr_distance_to_surface value over every primitive of every kind, prim[i] / geom[i] (may be
 * NULL) the primitive that gives it -- the first in the order triangles, spheres, planes,
 * cylinders and, within a kind, the lowest id among equal distances; +inf and BZR_INVALID_ID
 * when no primitive gives a number.  Triangles and spheres are searched through their BVHs
 * (a subtree is skipped only when its box is farther than the best distance), planes and
 * cylinders are evaluated one by one.  Arrays all host or all device memory, as above. */
int bzr_closest_surface(const bzr_scene *scene, size_t n, const double *points, double *distance,
                        uint32_t *prim, uint32_t *geom, void *stream);

/* Persistent scene format: a committed scene -- its inputs as added, build options and every
 * kind's BVH in the reference's node order -- as bytes, and a committed scene made from them
 * WITHOUT rebuilding the trees (the primitives' precompute is re-run; the trees are checked:
 * DFS structure, leaf lists a permutation of the primitives, node boxes equal to the unions of
 * their primitives' boxes; the bytes carry a checksum).  A loaded scene answers every query bit
 * for bit as the saved one.  The reference has no scene file (blazert/scene.h builds at every
 * commit).  bzr_scene_serialize returns the byte count (call with NULL to size the buffer) or a
 * negative status; damaged or inconsistent data is BZR_EINVAL with the reason in
 * bzr_last_error_string. */
long bzr_scene_serialize(const bzr_scene *scene, uint8_t *buffer, size_t capacity);
int bzr_scene_deserialize(bzr_scene **scene, const uint8_t *buffer, size_t size);
int bzr_scene_save(const bzr_scene *scene, const char *path);
int bzr_scene_load(bzr_scene **scene, const char *path);

/* Mesh ingestion: the vertices (n x 3) and triangles (m x 3) the reference's examples build
 * from a Wavefront OBJ file (examples/scene_mesh/main.cc:15-43 over the vendored
 * tiny_obj_loader 0.9.14, examples/common/tiny_obj_loader.cc:911-1081): the loader's own
 * number parser rounded to float, shapes ended by "g" and "o", vertices numbered per shape in
 * order of first use by (position, texcoord, normal) index triple, polygons split into fans,
 * shapes concatenated.  Ready for bzr_add_mesh.  The arrays are allocated here; release each
 * with bzr_obj_free.  A missing file or a face index outside the vertices is BZR_EINVAL. */
int bzr_obj_load(const char *path, double **vertices, size_t *n_vertices, uint32_t **faces,
                 size_t *n_faces);
void bzr_obj_free(void *p);

const char *bzr_last_error_string(void);

/* Test hook (no counterpart in the reference): the k-th device or pinned-host allocation this
 * library makes from now on fails as if the device were out of memory (k = 0 disarms; the
 * hook disarms itself when it fires).  The entry point that meets the failure returns
 * BZR_ENOMEM and releases what it had allocated; the scene stays usable. */
int bzr_debug_fail_allocation(int64_t k);

#ifdef __cplusplus
}
#endif
#endif /* BLAZERT_B200_H_ */
