"""ctypes loaders for the CPU checkers (TEST INFRASTRUCTURE ONLY).

* ``Oracle``   -- the plain-C restatement, ``oracle/liboracle.so`` (bzr_oracle.c).
* ``RefScene`` -- the reference's own headers compiled against the blaze shim,
  ``oracle/_ref/libref_parity.so`` (bit-exact build) or ``oracle/_ref/libref_bench.so``
  (release flags, the timed CPU baseline).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this module, and
only as the checker.  Both classes take a scene description with the same fields as the
product's ``blazert_b200.Scene`` (``SceneSpec`` in blazert_b200/workloads.py).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KINDS = ("mesh", "spheres", "planes", "cylinders")

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)
_ip = C.POINTER(C.c_int)


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(ctype)


def _f64(a, shape=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(shape) if shape is not None else a


def _u32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint32)


_CREATE_ARGS = [_ip, C.c_int, _dp, C.c_long, _u32p, C.c_long, _dp, _dp, C.c_long, _dp, _dp, _dp,
                _dp, C.c_long, _dp, _dp, _dp, _dp, _dp, C.c_long, C.c_uint, C.c_uint, C.c_uint,
                _u32p]
_TREE_ARGS = [C.c_void_p, C.c_int, _dp, _dp, _u32p, _u32p, _u32p, _u32p, _u32p, _u32p, C.c_long]


def _create_args(spec, opts):
    """Marshal a SceneSpec into the create() argument list shared by both libraries."""
    order = np.array([KINDS.index(k) for k in spec.order], dtype=np.int32)
    m, s, p, c = spec.mesh, spec.spheres, spec.planes, spec.cylinders
    keep = []

    def arr(x, conv):
        if x is None:
            return None
        y = conv(x)
        keep.append(y)
        return y

    verts = arr(m["vertices"] if m else None, lambda x: _f64(x).reshape(-1))
    faces = arr(m["faces"] if m else None, lambda x: _u32(x).reshape(-1))
    sc = arr(s["centers"] if s else None, lambda x: _f64(x).reshape(-1))
    sr = arr(s["radii"] if s else None, _f64)
    pc = arr(p["centers"] if p else None, lambda x: _f64(x).reshape(-1))
    pdx = arr(p["dxs"] if p else None, _f64)
    pdy = arr(p["dys"] if p else None, _f64)
    prot = arr(p["rotations"] if p else None, lambda x: _f64(x).reshape(-1))
    cc = arr(c["centers"] if c else None, lambda x: _f64(x).reshape(-1))
    ca = arr(c["semi_axes_a"] if c else None, _f64)
    cb = arr(c["semi_axes_b"] if c else None, _f64)
    ch = arr(c["heights"] if c else None, _f64)
    crot = arr(c["rotations"] if c else None, lambda x: _f64(x).reshape(-1))
    geom = np.full(len(order), 0xFFFFFFFF, dtype=np.uint32)
    keep += [order, geom]
    args = [_ptr(order, _ip), len(order),
            _ptr(verts, _dp), 0 if verts is None else verts.size // 3,
            _ptr(faces, _u32p), 0 if faces is None else faces.size // 3,
            _ptr(sc, _dp), _ptr(sr, _dp), 0 if sr is None else sr.size,
            _ptr(pc, _dp), _ptr(pdx, _dp), _ptr(pdy, _dp), _ptr(prot, _dp),
            0 if pdx is None else pdx.size,
            _ptr(cc, _dp), _ptr(ca, _dp), _ptr(cb, _dp), _ptr(ch, _dp), _ptr(crot, _dp),
            0 if ca is None else ca.size,
            opts[0], opts[1], opts[2], _ptr(geom, _u32p)]
    return args, keep, geom


class _Base:
    _lib = None
    _prefix = ""

    def __init__(self, spec, min_leaf=4, max_depth=28, bins=64):
        args, keep, geom = _create_args(spec, (min_leaf, max_depth, bins))
        self._h = getattr(self._lib, self._prefix + "scene_create")(*args)
        self._keep = keep
        self.geom_ids = {k: int(g) for k, g in zip(spec.order, geom)}

    def close(self):
        if getattr(self, "_h", None):
            getattr(self._lib, self._prefix + "scene_destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tree(self, kind):
        """Node arrays of one per-kind BVH, in the reference's node order."""
        k = KINDS.index(kind)
        f = getattr(self._lib, self._prefix + "scene_tree")
        n = f(self._h, k, None, None, None, None, None, None, None, None, 0)
        if n < 0:
            return None
        bmin = np.zeros((n, 3)); bmax = np.zeros((n, 3))
        leaf = np.zeros(n, np.uint32); axis = np.zeros(n, np.uint32)
        ch = np.zeros((n, 2), np.uint32); off = np.zeros(n, np.uint32)
        cnt = np.zeros(n, np.uint32)
        cap = 4 * n + 16
        prims = np.zeros(cap, np.uint32)
        f(self._h, k, _ptr(bmin, _dp), _ptr(bmax, _dp), _ptr(leaf, _u32p), _ptr(axis, _u32p),
          _ptr(ch, _u32p), _ptr(off, _u32p), _ptr(cnt, _u32p), _ptr(prims, _u32p), cap)
        total = int(cnt.sum())
        if total > cap:
            prims = np.zeros(total, np.uint32)
            f(self._h, k, _ptr(bmin, _dp), _ptr(bmax, _dp), _ptr(leaf, _u32p),
              _ptr(axis, _u32p), _ptr(ch, _u32p), _ptr(off, _u32p), _ptr(cnt, _u32p),
              _ptr(prims, _u32p), total)
        return dict(bmin=bmin, bmax=bmax, leaf=leaf, axis=axis, children=ch, prim_off=off,
                    prim_cnt=cnt, prim_ids=prims[:total])


_DIST_ARGS = [C.c_void_p, C.c_int, C.c_long, _u32p, _dp, _dp, _dp]
STAT_KEYS = ("max_tree_depth", "leaf_nodes", "max_num_prims_per_leaf", "min_num_prims_per_leaf",
             "branch_nodes", "bad_splits")
_NEAREST_ARGS = [C.c_void_p, C.c_long, _dp, _dp, _u32p, _u32p]


def _distance_to_surface(obj, kind, ids, points):
    ids = np.ascontiguousarray(ids, np.uint32).reshape(-1)
    pts = _f64(points).reshape(-1, 3)
    n = pts.shape[0]
    if ids.shape[0] != n:
        raise ValueError("one primitive id per point")
    dist = np.empty(n)
    closest = np.full((n, 3), np.nan)
    getattr(obj._lib, obj._prefix + "distance_to_surface")(
        obj._h, KINDS.index(kind), n, _ptr(ids, _u32p), _ptr(pts, _dp), _ptr(dist, _dp),
        _ptr(closest, _dp) if kind == "mesh" else None)
    return (dist, closest) if kind == "mesh" else (dist, None)


def _closest_surface(obj, points):
    pts = _f64(points).reshape(-1, 3)
    n = pts.shape[0]
    dist = np.empty(n)
    prim = np.empty(n, np.uint32)
    geom = np.empty(n, np.uint32)
    getattr(obj._lib, obj._prefix + "closest_surface")(obj._h, n, _ptr(pts, _dp),
                                                       _ptr(dist, _dp), _ptr(prim, _u32p),
                                                       _ptr(geom, _u32p))
    return dict(distance=dist, prim=prim, geom=geom)


def _outputs(n):
    return dict(t=np.empty(n), uv=np.empty((n, 2)), normal=np.empty((n, 3)),
                prim=np.empty(n, np.uint32), geom=np.empty(n, np.uint32),
                hit=np.empty(n, np.uint8))


def _rays(org, dirs, tmin, tmax):
    org = _f64(org).reshape(-1, 3)
    dirs = _f64(dirs).reshape(-1, 3)
    n = org.shape[0]
    tmin = None if tmin is None else np.ascontiguousarray(np.broadcast_to(tmin, (n,)), np.float64)
    tmax = None if tmax is None else np.ascontiguousarray(np.broadcast_to(tmax, (n,)), np.float64)
    return org, dirs, tmin, tmax, n


class Oracle(_Base):
    """The C restatement (bzr_oracle.c)."""

    _prefix = "ora_"

    @classmethod
    def load(cls):
        if cls._lib is None:
            path = os.path.join(HERE, "liboracle.so")
            if not os.path.exists(path):
                raise RuntimeError(f"{path} missing: run `make -C oracle` (or __graft_entry__.build())")
            lib = C.CDLL(path)
            lib.ora_scene_create.restype = C.c_void_p
            lib.ora_scene_create.argtypes = _CREATE_ARGS
            lib.ora_scene_destroy.argtypes = [C.c_void_p]
            lib.ora_scene_intersect.argtypes = [C.c_void_p, C.c_long, _dp, _dp, _dp, _dp, _dp, _dp,
                                                _dp, _u32p, _u32p, _u8p, _u32p, _u32p, C.c_int]
            lib.ora_scene_intersect_ex.argtypes = [C.c_void_p, C.c_long, _dp, _dp, _dp, _dp,
                                                   C.c_int, _dp, _dp, _dp, _u32p, _u32p, _u8p,
                                                   _u32p, _u32p, C.c_int]
            lib.ora_scene_tree.restype = C.c_long
            lib.ora_scene_tree.argtypes = _TREE_ARGS
            lib.ora_intersect_node.restype = C.c_int
            lib.ora_intersect_node.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp]
            lib.ora_intersect_primitive0.restype = C.c_int
            lib.ora_intersect_primitive0.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_double,
                                                     C.c_double, _dp, _dp, _dp, _u32p]
            lib.ora_traverse_kind.restype = C.c_int
            lib.ora_traverse_kind.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_double,
                                              C.c_double, _dp, _dp, _dp, _u32p]
            lib.ora_distance_to_surface.argtypes = _DIST_ARGS
            lib.ora_closest_surface.argtypes = _NEAREST_ARGS
            cls._lib = lib
        return cls._lib

    def __init__(self, spec, **kw):
        self.load()
        super().__init__(spec, **kw)

    def intersect(self, org, dirs, tmin=None, tmax=None, counters=False, nthreads=0,
                  any_hit=False):
        """intersect1 over the rays; any_hit: every ray with Ray::AnyHit::yes."""
        org, dirs, tmin, tmax, n = _rays(org, dirs, tmin, tmax)
        out = _outputs(n)
        cnt = np.zeros((n, 8), np.uint32) if counters else None
        peak = np.zeros(n, np.uint32) if counters else None
        self._lib.ora_scene_intersect_ex(
            self._h, n, _ptr(org, _dp), _ptr(dirs, _dp), _ptr(tmin, _dp), _ptr(tmax, _dp),
            1 if any_hit else 0, _ptr(out["t"], _dp), _ptr(out["uv"], _dp),
            _ptr(out["normal"], _dp), _ptr(out["prim"], _u32p), _ptr(out["geom"], _u32p),
            _ptr(out["hit"], _u8p), _ptr(cnt, _u32p), _ptr(peak, _u32p), nthreads)
        if counters:
            out["counters"] = cnt
            out["stack_peak"] = peak
        return out

    def primitive0(self, kind, org, d, tmin=0.0, tmax=np.finfo(np.float64).max):
        o = _f64(org); dd = _f64(d)
        t = np.zeros(1); uv = np.zeros(2); nrm = np.zeros(3); prim = np.zeros(1, np.uint32)
        h = self._lib.ora_intersect_primitive0(self._h, KINDS.index(kind), _ptr(o, _dp),
                                               _ptr(dd, _dp), tmin, tmax, _ptr(t, _dp),
                                               _ptr(uv, _dp), _ptr(nrm, _dp), _ptr(prim, _u32p))
        return dict(hit=bool(h), t=float(t[0]), uv=uv, normal=nrm, prim=int(prim[0]))

    def traverse(self, kind, org, d, tmin=0.0, tmax=np.finfo(np.float64).max):
        o = _f64(org); dd = _f64(d)
        t = np.zeros(1); uv = np.zeros(2); nrm = np.zeros(3); prim = np.zeros(1, np.uint32)
        h = self._lib.ora_traverse_kind(self._h, KINDS.index(kind), _ptr(o, _dp), _ptr(dd, _dp),
                                        tmin, tmax, _ptr(t, _dp), _ptr(uv, _dp), _ptr(nrm, _dp),
                                        _ptr(prim, _u32p))
        return dict(hit=bool(h), t=float(t[0]), uv=uv, normal=nrm, prim=int(prim[0]))

    def distance_to_surface(self, kind, ids, points):
        """(distances, closest points for meshes else None) of primitive ids[i] and point i."""
        return _distance_to_surface(self, kind, ids, points)

    def closest_surface(self, points):
        """Nearest surface over the whole scene, by exhaustion."""
        return _closest_surface(self, points)

    @classmethod
    def intersect_node(cls, tmin, tmax, bmin, bmax, org, raw_dir):
        lib = cls.load()
        a = np.array([tmin], np.float64); b = np.array([tmax], np.float64)
        h = lib.ora_intersect_node(_ptr(a, _dp), _ptr(b, _dp), _ptr(_f64(bmin), _dp),
                                   _ptr(_f64(bmax), _dp), _ptr(_f64(org), _dp),
                                   _ptr(_f64(raw_dir), _dp))
        return bool(h), float(a[0]), float(b[0])


class RefScene(_Base):
    """The reference's own headers (scene.h, bvh/, primitives/) compiled against the shim."""

    _prefix = "ref_"
    _libs = {}

    @classmethod
    def available(cls, flavour="parity"):
        return os.path.exists(os.path.join(HERE, "_ref", f"libref_{flavour}.so"))

    def __init__(self, spec, flavour="parity", **kw):
        if flavour not in RefScene._libs:
            path = os.path.join(HERE, "_ref", f"libref_{flavour}.so")
            if not os.path.exists(path):
                raise RuntimeError(f"{path} missing: build it with `make -C oracle ref`")
            lib = C.CDLL(path)
            lib.ref_scene_create.restype = C.c_void_p
            lib.ref_scene_create.argtypes = _CREATE_ARGS
            lib.ref_scene_destroy.argtypes = [C.c_void_p]
            lib.ref_scene_commit_seconds.restype = C.c_double
            lib.ref_scene_commit_seconds.argtypes = [C.c_void_p]
            lib.ref_scene_intersect.restype = C.c_double
            lib.ref_scene_intersect.argtypes = [C.c_void_p, C.c_long, _dp, _dp, _dp, _dp, _dp,
                                                _dp, _dp, _u32p, _u32p, _u8p, C.c_int]
            lib.ref_scene_intersect_ex.restype = C.c_double
            lib.ref_scene_intersect_ex.argtypes = [C.c_void_p, C.c_long, _dp, _dp, _dp, _dp,
                                                   C.c_int, _dp, _dp, _dp, _u32p, _u32p, _u8p,
                                                   C.c_int]
            lib.ref_scene_tree.restype = C.c_long
            lib.ref_scene_tree.argtypes = _TREE_ARGS
            lib.ref_scene_traverse_kind.restype = C.c_double
            lib.ref_scene_traverse_kind.argtypes = [C.c_void_p, C.c_int, C.c_long, _dp, _dp, _dp,
                                                    _u32p, _u8p, C.c_int]
            if hasattr(lib, "ref_distance_to_surface"):
                lib.ref_distance_to_surface.argtypes = _DIST_ARGS
            if hasattr(lib, "ref_build_statistics"):
                lib.ref_build_statistics.argtypes = [C.c_void_p, C.c_int, _u32p]
            RefScene._libs[flavour] = lib
        self._lib = RefScene._libs[flavour]
        super().__init__(spec, **kw)

    def build_statistics(self, kind):
        """The reference's BVHBuildStatistics of one kind (SAHBinnedBuilder::build's return)."""
        out = np.zeros(6, np.uint32)
        if self._lib.ref_build_statistics(self._h, KINDS.index(kind), _ptr(out, _u32p)) != 0:
            return None
        return dict(zip(STAT_KEYS, (int(x) for x in out)))

    def distance_to_surface(self, kind, ids, points):
        """The reference's own distance_to_surface (closest_point_on_triangle for meshes)."""
        return _distance_to_surface(self, kind, ids, points)

    @property
    def commit_seconds(self):
        return self._lib.ref_scene_commit_seconds(self._h)

    def intersect(self, org, dirs, tmin=None, tmax=None, nthreads=0, any_hit=False):
        """intersect1 over the rays; any_hit builds them with Ray::AnyHit::yes."""
        org, dirs, tmin, tmax, n = _rays(org, dirs, tmin, tmax)
        out = _outputs(n)
        secs = self._lib.ref_scene_intersect_ex(
            self._h, n, _ptr(org, _dp), _ptr(dirs, _dp), _ptr(tmin, _dp), _ptr(tmax, _dp),
            1 if any_hit else 0, _ptr(out["t"], _dp), _ptr(out["uv"], _dp),
            _ptr(out["normal"], _dp), _ptr(out["prim"], _u32p), _ptr(out["geom"], _u32p),
            _ptr(out["hit"], _u8p), nthreads)
        out["seconds"] = secs
        return out


def ref_load_obj(path):
    """(vertices, faces) of an OBJ file through the reference's vendored loader and the
    scene_mesh example's assembly (oracle/_ref/libref_obj.so); ValueError with the loader's
    message when it reports an error."""
    lib = C.CDLL(os.path.join(HERE, "_ref", "libref_obj.so"))
    lib.ref_obj_load.argtypes = [C.c_char_p, C.POINTER(C.POINTER(C.c_double)),
                                 C.POINTER(C.c_long), C.POINTER(C.POINTER(C.c_uint32)),
                                 C.POINTER(C.c_long), C.c_char_p, C.c_long]
    lib.ref_obj_free.argtypes = [C.c_void_p]
    pv, pf = C.POINTER(C.c_double)(), C.POINTER(C.c_uint32)()
    nv, nf = C.c_long(), C.c_long()
    why = C.create_string_buffer(512)
    if lib.ref_obj_load(os.fsencode(path), C.byref(pv), C.byref(nv), C.byref(pf), C.byref(nf),
                        why, 512):
        raise ValueError(why.value.decode(errors="replace"))
    try:
        v = np.ctypeslib.as_array(pv, (3 * nv.value + 1,))[: 3 * nv.value].reshape(-1, 3).copy()
        f = np.ctypeslib.as_array(pf, (3 * nf.value + 1,))[: 3 * nf.value].reshape(-1, 3).copy()
    finally:
        lib.ref_obj_free(C.cast(pv, C.c_void_p))
        lib.ref_obj_free(C.cast(pf, C.c_void_p))
    return v, f
