// Device data layout shared by the host flattener (scene.cpp) and the kernels (trace.cu).
//
// One BVH per primitive kind, as in the reference (blazert/scene.h:52-70).  The reference's
// binary tree (blazert/bvh/node.h:15-41: each node holds its own box; leaves hold a vector of
// primitives) is re-laid out for the GPU:
//
//  * Only INTERNAL nodes become device nodes, numbered breadth-first (so the top levels are a
//    contiguous prefix).  A device node holds the boxes of its two CHILDREN, so one 128-byte
//    line gives both slab tests, and a child is never fetched just to be rejected.
//  * A child reference is either a device-node index, or kLeafBit | q where q is the position
//    of the leaf's first primitive in the leaf-ordered primitive arrays.  The leaf's primitives
//    follow contiguously in the reference's stored order (blazert/bvh/builder.h:133-148); the
//    last one carries kLastBit in its id word.
//  * The root's own box and reference live in KindView (the reference tests the root box
//    first, blazert/bvh/accel.h:83-97).
#pragma once
#include <cstdint>

namespace bzr {

constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kLastBit = 0x80000000u;
constexpr uint32_t kIdMask = 0x7FFFFFFFu;

enum Kind : int { kMesh = 0, kSpheres = 1, kPlanes = 2, kCylinders = 3, kNumKinds = 4 };

// FP64 node, 16 doubles = 128 bytes (8 x 16-byte loads):
//   d[0..5]   child 0: (lo.x, hi.x), (lo.y, hi.y), (lo.z, hi.z)
//   d[6..11]  child 1: same
//   d[12..13] uint32 {ref0, ref1, axis, 0}
//   d[14..15] unused
constexpr int kNode64Doubles = 16;

// Leaf-ordered primitive payload, doubles per primitive:
//   spheres     4: center(3), radius
//   planes     14: center(3), dx, dy, rotation(9, row-major)
//   cylinders  16: center(3), semi_axis_a, semi_axis_b, height, rotation(9), pad
// Triangles are indexed instead (the reference's TriangleMesh keeps vertices and faces,
// blazert/primitives/trimesh.h:78-90, and builds v0, e1 = v0 - v1, e2 = v2 - v0 per test,
// trimesh.h:153-160): per leaf-ordered triangle one 16-byte word group {i0, i1, i2, id word}
// indexing a vertex array of 32-byte {x, y, z, 0} entries, the vertices numbered in order of
// first use by the leaf-ordered triangles (so a leaf's vertices sit together) and each shared
// vertex stored once.  That is 16 B + 3 x 32 B per test against 96 B for a precomputed
// record, but the distinct data of a mesh is 16 B per triangle + 32 B per vertex: a 2M-triangle
// grid needs 67 MB instead of 201 MB, which keeps far more of it in L2.
constexpr int kPayloadDoubles[kNumKinds] = {0, 4, 14, 16};
constexpr int kVertexDoubles = 4;

// Mixed-precision image (triangles, spheres, planes; BZR_MODE_MIXED).  The reference's binary
// tree is cut into treelets of up to kWideMax children -- from an internal node, the internal
// child of largest box surface is replaced by its two children until the treelet has
// kWideMax children or only leaves -- and each treelet becomes one 128-byte wide node whose
// children's boxes are stored as 8-bit integers on a per-axis grid of spacing 2^e, rounded
// outward, so every stored box contains the child's exact box:
//   bytes  0..11  float origin[3]: k_a * 2^e_a, exactly representable (|k_a| < 2^24)
//   bytes 12..15  u32 e_x + 127 | (e_y + 127) << 8 | (e_z + 127) << 16 | children << 24
//   bytes 16..63  u8: for axis a, lo[8] at 16 + 16a and hi[8] at 24 + 16a; child c's box on
//                 axis a is [origin + lo[c] * 2^e, origin + hi[c] * 2^e]; an unused slot has
//                 lo = 255, hi = 0 (an empty box)
//   bytes 64..95  u32 ref[8]: a wide node index, or kLeafBit | a leaf record's offset in
//                 16-byte units
//   bytes 96..127 u32 perm[8]: for a ray of direction-sign octant s = sx | sy << 1 | sz << 2,
//                 nibble j of perm[s] is the slot of the j-th child in the reference's visit
//                 order, 15 past the last child (the reference visits
//                 children[direction_sign[axis]] first at every binary node,
//                 blazert/bvh/accel.h:100-104, so a treelet's order depends on s only).
// Leaf records (16-byte aligned): the leaf's exact FP64 box (lo.x, hi.x, lo.y, hi.y, lo.z,
// hi.z; 48 B), u32 first leaf-ordered position, u32 count, 8 B zero; then the leaf's
// primitives: triangles {i0, i1, i2, 0} (16 B, indices into the vertex array), spheres and
// planes their payload records (32 B, 112 B).
constexpr int kWideMax = 8;
// Entries of the thread-local traversal stack; trees whose stack needs more (depth > 62,
// reachable only with max_tree_depth above 62) trace with the stack in shared memory in FP64,
// and a kind whose wide traversal could need more has no mixed-precision image.
constexpr uint32_t kLocalStack = 64;
constexpr int kWideBytes = 128;
constexpr int kLeafHeaderBytes = 64;

struct KindView {
  const double *nodes64 = nullptr;  // n_internal * kNode64Doubles
  const double *payload = nullptr;  // n_prims * kPayloadDoubles[kind] (spheres, planes, cylinders)
  const uint32_t *tri = nullptr;    // triangles: n_prims * 4 {i0, i1, i2, id word}
  const double *verts = nullptr;    // triangles: kVertexDoubles per vertex {x, y, z, 0}
  const double *vnorm = nullptr;    // triangles: kVertexDoubles per vertex of verts: its vertex
                                    // normal {nx, ny, nz, 0}
  const uint32_t *prim_ids = nullptr;  // n_prims: id | kLastBit on a leaf's last primitive
  const uint32_t *pos_of = nullptr;    // n_prims: leaf-ordered position of each primitive id
  uint32_t n_internal = 0;
  uint32_t n_prims = 0;
  uint32_t n_verts = 0;             // triangles: entries of verts
  uint32_t root_ref = 0;
  uint32_t geom_id = 0xFFFFFFFFu;
  int present = 0;
  int mixed_ok = 0;                 // wide image present: the FP32 path may be used
  double root_box[6] = {0, 0, 0, 0, 0, 0};  // (lo.x, hi.x, lo.y, hi.y, lo.z, hi.z)
  // mixed-precision image (see kWideBytes); the root's wide node is index 0
  const unsigned char *wide = nullptr;   // n_wide * kWideBytes
  const double *leaves = nullptr;        // leaf records, n_leaf16 16-byte units
  uint32_t n_wide = 0;
  uint32_t n_leaf16 = 0;
  uint32_t wide_root_ref = 0;            // 0 (wide root) or kLeafBit | offset of a leaf root
  float coord_max = 0.0f;       // largest |coordinate| of the root box, rounded up
};

struct SceneView {
  KindView k[kNumKinds];
  const uint32_t *faces = nullptr;   // n_faces * 3, original order (triangle normals)
  const double *vert_n = nullptr;    // n_vertices * 3 accumulated vertex normals
  uint32_t stack_cap = 32;           // traversal stack entries per thread
};

// Kernel error word bits.
constexpr uint32_t kErrStack = 1u;      // traversal stack would overflow
constexpr uint32_t kErrNodeIndex = 2u;  // a child reference points outside the node array
constexpr uint32_t kErrPrimIndex = 4u;  // a leaf runs past the primitive arrays
constexpr uint32_t kErrAdjointKind = 8u;  // a ray's hit kind has no adjoint (plane, cylinder)

}  // namespace bzr
