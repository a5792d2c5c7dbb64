// Persistent scene format: a committed scene written to bytes and read back without rebuilding
// its BVHs.  The reference keeps no scene on disk (blazert/scene.h builds at every commit);
// this is the checkpoint of the query path: the inputs as they were added, the build options
// and each kind's tree in the reference's DFS node order (blazert/bvh/node.h:15-41) with its
// leaf primitive list.  Reading it re-runs the collections' precompute (boxes, centres,
// normals; deterministic), attaches the stored trees after checking them, and the caller
// flattens and uploads as a commit does -- so a loaded scene answers every query bit for bit
// as the scene that was saved.
//
// Layout (little endian):
//   "BZRSCENE" | u32 version (1) | u32 min_leaf, max_depth, bins | u32 n_kinds
//   n_kinds x { u32 kind, u32 geom_id, u64 n, the kind's input arrays, the tree }
//   u64 hash of every byte before it
// The hash of version 2 (written): the bytes before it cut into blocks of 2^20 bytes (the last
// one shorter), each block hashed with 64-bit FNV-1a, then FNV-1a over the little-endian u64
// block hashes in order; the blocks are hashed on several threads.  Version 1 (still read) is
// FNV-1a over all those bytes at once and otherwise the same format.
// Input arrays: mesh u64 n_vertices, f64 vertices[3 nv], u32 faces[3 n]; spheres centres[3n],
// radii[n]; planes centres[3n], dxs[n], dys[n], rotations[9n]; cylinders centres[3n], a[n],
// b[n], heights[n], rotations[9n].  Tree: u64 n_nodes, per node f64 min[3], max[3], u32 leaf,
// axis, child0, child1, prim_off, prim_cnt; u64 n_leaf_prims, u32 leaf_prims[]; u32 bad_splits.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "scene.h"

namespace bzr {
namespace {

constexpr char kMagic[8] = {'B', 'Z', 'R', 'S', 'C', 'E', 'N', 'E'};
constexpr uint32_t kVersion = 2;       // written
constexpr uint32_t kVersionWhole = 1;  // read: one FNV-1a over all the bytes
constexpr size_t kHashBlock = size_t(1) << 20;
constexpr size_t kNodeBytes = 6 * sizeof(double) + 6 * sizeof(uint32_t);  // one tree node

uint64_t fnv1a(const uint8_t *p, size_t n) {
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

// The version-2 hash of n bytes (see the layout above).
uint64_t block_hash(const uint8_t *p, size_t n) {
  const size_t nb = (n + kHashBlock - 1) / kHashBlock;
  std::vector<uint8_t> hashes(8 * nb);
  run_ranges(nb, range_workers(nb, 4, 16), [&](size_t b0, size_t b1, size_t) {
    for (size_t b = b0; b < b1; ++b) {
      const uint64_t h = fnv1a(p + b * kHashBlock, std::min(kHashBlock, n - b * kHashBlock));
      for (int i = 0; i < 8; ++i) hashes[8 * b + i] = static_cast<uint8_t>(h >> (8 * i));
    }
  });
  return fnv1a(hashes.data(), hashes.size());
}

struct Writer {
  RawVector<uint8_t> out;  // grow() writes every byte it appends
  // appends `bytes` bytes and returns where they start
  uint8_t *grow(size_t bytes) {
    const size_t at = out.size();
    out.resize(at + bytes);
    return out.data() + at;
  }
  template <class T>
  void put(const T &v) {
    std::memcpy(grow(sizeof(T)), &v, sizeof(T));
  }
  template <class T>
  void put_array(const T *p, size_t n) {
    if (n) std::memcpy(grow(n * sizeof(T)), p, n * sizeof(T));
  }
};

struct Reader {
  const uint8_t *p;
  size_t n, at = 0;
  bool ok = true;
  template <class T>
  T get() {
    T v{};
    if (!ok || n - at < sizeof(T)) {
      ok = false;
      return v;
    }
    std::memcpy(&v, p + at, sizeof(T));
    at += sizeof(T);
    return v;
  }
  template <class T>
  bool get_array(std::vector<T> &v, uint64_t count) {
    if (!ok || count > (n - at) / sizeof(T)) return ok = false;
    v.resize(count);
    if (count) std::memcpy(v.data(), p + at, count * sizeof(T));
    at += count * sizeof(T);
    return true;
  }
};

void put_tree(Writer &w, const Tree &t) {
  w.put<uint64_t>(t.nodes.size());
  uint8_t *p = w.grow(t.nodes.size() * kNodeBytes);
  for (const TreeNode &nd : t.nodes) {
    const uint32_t u[6] = {nd.leaf, nd.axis, nd.child[0], nd.child[1], nd.prim_off, nd.prim_cnt};
    std::memcpy(p, nd.mn, sizeof nd.mn);
    std::memcpy(p + sizeof nd.mn, nd.mx, sizeof nd.mx);
    std::memcpy(p + sizeof nd.mn + sizeof nd.mx, u, sizeof u);
    p += kNodeBytes;
  }
  w.put<uint64_t>(t.leaf_prims.size());
  w.put_array(t.leaf_prims.data(), t.leaf_prims.size());
  w.put<uint32_t>(t.bad_splits);
}

// Bytes encode_scene writes for the kinds order[0..n_kinds), the hash included.
size_t encoded_size(const HostScene &s, const uint32_t *order, int n_kinds) {
  size_t bytes = 8 + 4 + 3 * 4 + 4 + 8;
  for (int j = 0; j < n_kinds; ++j) {
    const Collection &c = s.kind[order[j]];
    bytes += 4 + 4 + 8;
    switch (order[j]) {
      case kMesh:
        bytes += 8 + s.vertices.size() * sizeof(double) + s.faces.size() * sizeof(uint32_t);
        break;
      case kSpheres:
        bytes += 4 * c.n * sizeof(double);
        break;
      case kPlanes:
        bytes += 14 * c.n * sizeof(double);
        break;
      case kCylinders:
        bytes += 15 * c.n * sizeof(double);
        break;
    }
    bytes += 8 + c.tree.nodes.size() * kNodeBytes + 8 + c.tree.leaf_prims.size() * 4 + 4;
  }
  return bytes;
}

bool finite_boxes(const PrimBoxes &b) {
  for (size_t i = 0; i < 3 * b.n; ++i)
    if (!std::isfinite(b.bmin[i]) || !std::isfinite(b.bmax[i])) return false;
  return true;
}

// Structure of a tree read from a file against its collection: DFS pre-order (the left child
// right after its parent, the right child after the left subtree), leaf ranges tiling the
// leaf list left to right, the leaf list a permutation of the primitives, depth within the
// options' limit; and, when every primitive box is finite, every node box equal (by value) to
// the union of the boxes under it, which is what the builder computes.  Sets max_depth.
std::string check_tree(Tree &t, const PrimBoxes &boxes, const BuildOptions &opt) {
  const size_t nn = t.nodes.size(), n = boxes.n;
  if (n == 0) {  // an empty collection: at most its one empty leaf
    if (nn > 1 || !t.leaf_prims.empty()) return "nodes of an empty collection";
    t.max_depth = 0;
    return "";
  }
  if (nn == 0 || nn > 2 * n + 1) return "node count does not fit the primitive count";
  if (t.leaf_prims.size() != n) return "leaf list length differs from the primitive count";
  std::vector<uint8_t> seen(n, 0);
  for (uint32_t id : t.leaf_prims) {
    if (id >= n || seen[id]) return "leaf list is not a permutation of the primitives";
    seen[id] = 1;
  }
  std::vector<uint32_t> depth(nn, 0);
  uint64_t next_prim = 0;
  uint32_t max_depth = 0;
  for (size_t i = 0; i < nn; ++i) {
    const TreeNode &nd = t.nodes[i];
    max_depth = depth[i] > max_depth ? depth[i] : max_depth;
    if (nd.leaf == 1) {
      if (nd.prim_off != next_prim || nd.prim_cnt == 0 || nd.prim_cnt > n - next_prim)
        return "leaf ranges do not tile the leaf list";
      next_prim += nd.prim_cnt;
    } else if (nd.leaf == 0) {
      if (nd.child[0] != i + 1 || nd.child[1] <= i + 1 || nd.child[1] >= nn || nd.axis > 2)
        return "node links are not a DFS pre-order";
      depth[nd.child[0]] = depth[i] + 1;
      depth[nd.child[1]] = depth[i] + 1;
    } else {
      return "bad leaf flag";
    }
  }
  if (next_prim != n) return "leaf ranges do not cover the leaf list";
  // the right child must start right after the left subtree: walk the subtree sizes
  std::vector<uint32_t> size(nn, 1);
  for (size_t i = nn; i-- > 0;) {
    const TreeNode &nd = t.nodes[i];
    if (nd.leaf == 0) {
      if (nd.child[1] != i + 1 + size[i + 1]) return "node links are not a DFS pre-order";
      size[i] = 1 + size[nd.child[0]] + size[nd.child[1]];
    }
  }
  if (size[0] != nn) return "nodes outside the tree";
  if (max_depth > opt.max_depth) return "tree deeper than its build options allow";
  if (finite_boxes(boxes)) {
    // A leaf's box against the union of its primitives' boxes, an internal node's against the
    // union of its children's stored boxes: with every node checked, this holds exactly when
    // every node box equals (by value) the union of the primitive boxes under it.
    for (size_t i = 0; i < nn; ++i) {
      const TreeNode &nd = t.nodes[i];
      double l[3], h[3];
      if (nd.leaf == 1) {
        for (int a = 0; a < 3; ++a) {
          l[a] = boxes.bmin[3 * size_t(t.leaf_prims[nd.prim_off]) + a];
          h[a] = boxes.bmax[3 * size_t(t.leaf_prims[nd.prim_off]) + a];
        }
        for (uint32_t q = 1; q < nd.prim_cnt; ++q) {
          const size_t id = t.leaf_prims[nd.prim_off + q];
          for (int a = 0; a < 3; ++a) {
            l[a] = std::fmin(l[a], boxes.bmin[3 * id + a]);
            h[a] = std::fmax(h[a], boxes.bmax[3 * id + a]);
          }
        }
      } else {
        const TreeNode &c0 = t.nodes[nd.child[0]], &c1 = t.nodes[nd.child[1]];
        for (int a = 0; a < 3; ++a) {
          l[a] = std::fmin(c0.mn[a], c1.mn[a]);
          h[a] = std::fmax(c0.mx[a], c1.mx[a]);
        }
      }
      for (int a = 0; a < 3; ++a)
        if (nd.mn[a] != l[a] || nd.mx[a] != h[a]) return "node box differs from its primitives";
    }
  }
  t.max_depth = max_depth;
  return "";
}

}  // namespace

RawVector<uint8_t> encode_scene(const HostScene &s) {
  // kinds in add order (their geom ids)
  uint32_t order[kNumKinds];
  int n_kinds = 0;
  for (uint32_t g = 0; g < kNumKinds; ++g)
    for (int k = 0; k < kNumKinds; ++k)
      if (s.kind[k].present && s.kind[k].geom_id == g) order[n_kinds++] = static_cast<uint32_t>(k);
  Writer w;
  w.out.reserve(encoded_size(s, order, n_kinds));
  w.put_array(kMagic, 8);
  w.put<uint32_t>(kVersion);
  w.put<uint32_t>(s.opt.min_leaf);
  w.put<uint32_t>(s.opt.max_depth);
  w.put<uint32_t>(s.opt.bins);
  w.put<uint32_t>(static_cast<uint32_t>(n_kinds));
  for (int j = 0; j < n_kinds; ++j) {
    const int k = static_cast<int>(order[j]);
    const Collection &c = s.kind[k];
    w.put<uint32_t>(static_cast<uint32_t>(k));
    w.put<uint32_t>(c.geom_id);
    w.put<uint64_t>(c.n);
    switch (k) {
      case kMesh:
        w.put<uint64_t>(s.vertices.size() / 3);
        w.put_array(s.vertices.data(), s.vertices.size());
        w.put_array(s.faces.data(), s.faces.size());
        break;
      case kSpheres:
        w.put_array(c.a.data(), 3 * c.n);
        w.put_array(c.b.data(), c.n);
        break;
      case kPlanes:
        w.put_array(c.a.data(), 3 * c.n);
        w.put_array(c.b.data(), c.n);
        w.put_array(c.c.data(), c.n);
        w.put_array(c.d.data(), 9 * c.n);
        break;
      case kCylinders:
        w.put_array(c.a.data(), 3 * c.n);
        w.put_array(c.b.data(), c.n);
        w.put_array(c.c.data(), c.n);
        w.put_array(c.d.data(), c.n);
        w.put_array(c.e.data(), 9 * c.n);
        break;
    }
    put_tree(w, c.tree);
  }
  w.put<uint64_t>(block_hash(w.out.data(), w.out.size()));
  return std::move(w.out);
}

std::string decode_scene(const uint8_t *data, size_t size, HostScene *out) {
  uint32_t order[kNumKinds] = {0, 0, 0, 0};
  if (size < 8 + 4 + 8 || std::memcmp(data, kMagic, 8) != 0) return "not a scene file";
  uint64_t stored = 0;
  std::memcpy(&stored, data + size - 8, 8);
  uint32_t version = 0;
  std::memcpy(&version, data + 8, 4);
  if (version != kVersion && version != kVersionWhole) return "unsupported scene file version";
  const uint64_t hash = version == kVersion ? block_hash(data, size - 8) : fnv1a(data, size - 8);
  if (hash != stored) return "checksum mismatch (damaged file)";
  Reader r{data, size - 8};
  r.at = 12;
  HostScene &s = *out;
  s = HostScene();
  s.opt.min_leaf = r.get<uint32_t>();
  s.opt.max_depth = r.get<uint32_t>();
  s.opt.bins = r.get<uint32_t>();
  const uint32_t nk = r.get<uint32_t>();
  if (!r.ok || nk > kNumKinds) return "bad kind count";
  if (s.opt.bins < 2 || s.opt.max_depth > 1000) return "bad build options";
  for (uint32_t j = 0; j < nk; ++j) {
    const uint32_t k = r.get<uint32_t>();
    const uint32_t geom = r.get<uint32_t>();
    const uint64_t n = r.get<uint64_t>();
    if (!r.ok || k >= kNumKinds || s.kind[k].present) return "bad kind record";
    if (n > 0x7FFFFFFFu) return "primitive count too large";
    std::vector<double> a, b, c, d, e;
    std::vector<uint32_t> f;
    switch (k) {
      case kMesh: {
        const uint64_t nv = r.get<uint64_t>();
        if (!r.ok || nv > 0xFFFFFFFFu) return "bad vertex count";
        if (!r.get_array(a, 3 * nv) || !r.get_array(f, 3 * n)) return "truncated mesh";
        for (uint32_t x : f)
          if (x >= nv) return "face index outside the vertices";
        add_mesh(s, a.data(), nv, f.data(), n);
        break;
      }
      case kSpheres:
        if (!r.get_array(a, 3 * n) || !r.get_array(b, n)) return "truncated spheres";
        add_spheres(s, a.data(), b.data(), n);
        break;
      case kPlanes:
        if (!r.get_array(a, 3 * n) || !r.get_array(b, n) || !r.get_array(c, n) ||
            !r.get_array(d, 9 * n))
          return "truncated planes";
        add_planes(s, a.data(), b.data(), c.data(), d.data(), n);
        break;
      default:
        if (!r.get_array(a, 3 * n) || !r.get_array(b, n) || !r.get_array(c, n) ||
            !r.get_array(d, n) || !r.get_array(e, 9 * n))
          return "truncated cylinders";
        add_cylinders(s, a.data(), b.data(), c.data(), d.data(), e.data(), n);
        break;
    }
    Collection &col = s.kind[k];
    col.present = true;
    col.geom_id = geom;
    const uint64_t nn = r.get<uint64_t>();
    if (!r.ok || nn > 2 * n + 1) return "bad node count";
    if (nn > (r.n - r.at) / kNodeBytes) return "truncated tree";
    Tree t;
    t.nodes.resize(nn);
    const uint8_t *q = r.p + r.at;
    for (TreeNode &nd : t.nodes) {
      uint32_t u[6];
      std::memcpy(nd.mn, q, sizeof nd.mn);
      std::memcpy(nd.mx, q + sizeof nd.mn, sizeof nd.mx);
      std::memcpy(u, q + sizeof nd.mn + sizeof nd.mx, sizeof u);
      nd.leaf = u[0];
      nd.axis = u[1];
      nd.child[0] = u[2];
      nd.child[1] = u[3];
      nd.prim_off = u[4];
      nd.prim_cnt = u[5];
      q += kNodeBytes;
    }
    r.at += nn * kNodeBytes;
    const uint64_t nl = r.get<uint64_t>();
    if (!r.ok || nl != n || !r.get_array(t.leaf_prims, nl)) return "truncated tree";
    t.bad_splits = r.get<uint32_t>();
    if (!r.ok) return "truncated tree";
    const std::string why = check_tree(t, col.boxes, s.opt);
    if (!why.empty()) return "tree of kind " + std::to_string(k) + ": " + why;
    col.tree = std::move(t);
    order[j] = k;
  }
  if (r.at != r.n) return "trailing bytes";
  // geom ids are the add order 0, 1, ...: unique and below the kind count
  uint32_t used = 0;
  for (uint32_t j = 0; j < nk; ++j) {
    const uint32_t g = s.kind[order[j]].geom_id;
    if (g >= nk || (used >> g) & 1u) return "bad geometry ids";
    used |= 1u << g;
  }
  s.geometries = nk;
  return "";
}

}  // namespace bzr
