"""blazert_b200 -- blazeRT's closest-hit ray query on B200, behind blazeRT's Scene API.

Python mirror of the reference interface (blazert/scene.h, blazert/ray.h) over the C-ABI of
``libblazert_b200.so`` (include/blazert_b200.h):

    scene = Scene()
    gid = scene.add_mesh(vertices, faces)          # BlazertScene::add_mesh, scene.h:227-240
    scene.add_spheres(centers, radii)              # scene.h:258-271
    scene.add_planes(centers, dxs, dys, rotations) # scene.h:293-307
    scene.add_cylinders(centers, a, b, heights, rotations)   # scene.h:331-346
    scene.commit()                                 # scene.h:91-115
    hit = intersect1(scene, Ray(origin, direction), rayhit)  # scene.h:161-210
    out = scene.intersectN(origins, directions)    # batched, one GPU launch

As in the reference, ``add_*`` returns the geom id, or ``INVALID_ID`` (the reference's
``static_cast<unsigned>(-1)``) when the kind was already added or the scene is committed.
Errors other than that raise ``BlazertError``.  There is no CPU fallback: without the built
library or a CUDA device the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libblazert_b200.so")

INVALID_ID = 0xFFFFFFFF
DBL_MAX = float(np.finfo(np.float64).max)
MODES = {"fp64": 0, "mixed": 1}
RAY_ANY_HIT = 1  # BZR_RAY_ANY_HIT

OK, EINVAL, ESTATE, ENOMEM, ECUDA, ETIMEOUT, EDEVICE_FLAG, ENODEV = 0, -1, -2, -3, -4, -5, -6, -7


class BlazertError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} (status {code})")
        self.code = code


_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)


class _RayHitC(C.Structure):
    _fields_ = [("normal", C.c_double * 3), ("uv", C.c_double * 2), ("hit_distance", C.c_double),
                ("prim_id", C.c_uint32), ("geom_id", C.c_uint32)]


class _OptsC(C.Structure):
    _fields_ = [("min_leaf_primitives", C.c_uint32), ("max_tree_depth", C.c_uint32),
                ("bin_size", C.c_uint32)]


_lib = None


def library():
    """Loads libblazert_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BlazertError(ENODEV, f"{LIB_PATH} is missing: run `python -m blazert_b200.build`")
        lib = C.CDLL(LIB_PATH)
        P = C.c_void_p
        lib.bzr_scene_create.argtypes = [C.POINTER(P)]
        lib.bzr_scene_destroy.argtypes = [P]
        lib.bzr_add_mesh.argtypes = [P, _dp, C.c_size_t, _u32p, C.c_size_t, _u32p]
        lib.bzr_add_spheres.argtypes = [P, _dp, _dp, C.c_size_t, _u32p]
        lib.bzr_add_planes.argtypes = [P, _dp, _dp, _dp, _dp, C.c_size_t, _u32p]
        lib.bzr_add_cylinders.argtypes = [P, _dp, _dp, _dp, _dp, _dp, C.c_size_t, _u32p]
        lib.bzr_commit.argtypes = [P, C.POINTER(_OptsC)]
        lib.bzr_intersect1.argtypes = [P, _dp, _dp, C.c_double, C.c_double,
                                       C.POINTER(_RayHitC), C.POINTER(C.c_int)]
        lib.bzr_intersectN.argtypes = [P, C.c_size_t, P, P, P, P, P, P, P, P, P, P, C.c_int, P]
        lib.bzr_intersect1_ex.argtypes = [P, _dp, _dp, C.c_double, C.c_double, C.c_uint32,
                                          C.POINTER(_RayHitC), C.POINTER(C.c_int)]
        lib.bzr_intersectN_ex.argtypes = [P, C.c_size_t, P, P, P, P, P, P, P, P, P, P, C.c_int,
                                          C.c_uint32, P]
        lib.bzr_scene_check.argtypes = [P, P, C.c_int, _u32p]
        lib.bzr_work_counts.argtypes = [P, C.c_size_t, P, P, P, P, C.POINTER(C.c_uint64), P]
        lib.bzr_work_counts_ex.argtypes = [P, C.c_size_t, P, P, P, P, C.c_int,
                                           C.POINTER(C.c_uint64), P]
        lib.bzr_scene_tune.argtypes = [P, C.c_int, C.c_int64]
        lib.bzr_adjoint_hit.argtypes = [P, C.c_size_t] + [P] * 14 + [P]
        lib.bzr_batch_create.argtypes = [C.POINTER(P), C.POINTER(P), C.c_size_t]
        lib.bzr_batch_destroy.argtypes = [P]
        lib.bzr_batch_intersect.argtypes = [P, C.POINTER(C.c_uint64)] + [P] * 11 + [C.c_int, P]
        lib.bzr_batch_check.argtypes = [P, P, _u32p]
        lib.bzr_batch_tune.argtypes = [P, C.c_int, C.c_int64]
        lib.bzr_commit_ex.argtypes = [P, C.POINTER(_OptsC), C.c_uint32]
        lib.bzr_scene_tree.restype = C.c_long
        lib.bzr_scene_tree.argtypes = [P, C.c_int] + [P] * 7 + [C.c_long]
        lib.bzr_scene_stats.argtypes = [P, C.c_int, C.POINTER(C.c_uint64), _u32p,
                                        C.POINTER(C.c_double)]
        lib.bzr_distance_to_surface.argtypes = [P, C.c_int, C.c_size_t, P, P, P, P, P]
        lib.bzr_closest_surface.argtypes = [P, C.c_size_t, P, P, P, P, P]
        lib.bzr_scene_serialize.restype = C.c_long
        lib.bzr_scene_serialize.argtypes = [P, P, C.c_size_t]
        lib.bzr_scene_deserialize.argtypes = [C.POINTER(P), P, C.c_size_t]
        lib.bzr_scene_save.argtypes = [P, C.c_char_p]
        lib.bzr_scene_load.argtypes = [C.POINTER(P), C.c_char_p]
        lib.bzr_obj_load.argtypes = [C.c_char_p, C.POINTER(C.POINTER(C.c_double)),
                                     C.POINTER(C.c_size_t), C.POINTER(C.POINTER(C.c_uint32)),
                                     C.POINTER(C.c_size_t)]
        lib.bzr_obj_free.argtypes = [P]
        lib.bzr_scene_build_statistics.argtypes = [P, C.c_int, P]
        lib.bzr_last_error_string.restype = C.c_char_p
        _lib = lib
    return _lib


KIND_NAMES = ("mesh", "spheres", "planes", "cylinders")


def _is_cuda_tensor(a):
    try:
        import torch
    except ImportError:
        return False
    return isinstance(a, torch.Tensor) and a.is_cuda


def _check(rc):
    if rc != OK:
        raise BlazertError(rc, library().bzr_last_error_string().decode())


def _f64(a, cols=None):
    """float64, C-contiguous; with cols, n x cols.  Accepts flat arrays (a multiple of cols
    values) and arrays whose rows hold cols values (n x 3 points; n x 3 x 3 or n x 9 rotations,
    or one 3 x 3 rotation); anything else is refused rather than silently reshaped."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    if not cols:
        return a.reshape(-1)
    if a.ndim >= 2 and int(np.prod(a.shape[1:])) != cols and not (cols == 9 and a.shape == (3, 3)):
        raise ValueError(f"expected rows of {cols} values, got an array of shape {a.shape}")
    if a.ndim <= 1 and a.size % cols:
        raise ValueError(f"expected a multiple of {cols} values, got {a.size}")
    return a.reshape(-1, cols)


@dataclass
class Ray:
    """blazert/ray.h:56-65.  The direction need not be unit length.  any_hit is the reference's
    Ray::AnyHit::yes: each kind's traversal stops at its first accepted hit (shadow rays)."""

    origin: np.ndarray
    direction: np.ndarray
    min_hit_distance: float = 0.0
    max_hit_distance: float = DBL_MAX
    any_hit: bool = False


@dataclass
class RayHit:
    """blazert/ray.h:72-85, with the reference's defaults for a miss."""

    normal: np.ndarray = field(default_factory=lambda: np.zeros(3))
    uv: np.ndarray = field(default_factory=lambda: np.zeros(2))
    hit_distance: float = DBL_MAX
    prim_id: int = INVALID_ID
    geom_id: int = INVALID_ID


@dataclass
class BuildOptions:
    """blazert/bvh/options.h:15-29."""

    min_leaf_primitives: int = 4
    max_tree_depth: int = 28
    bin_size: int = 64


def load_obj(path):
    """(vertices n x 3 float64, faces m x 3 uint32) of a Wavefront OBJ file, as the reference's
    examples build the mesh (bzr_obj_load); ready for Scene.add_mesh."""
    lib = library()
    pv, pf = C.POINTER(C.c_double)(), C.POINTER(C.c_uint32)()
    nv, nf = C.c_size_t(), C.c_size_t()
    _check(lib.bzr_obj_load(os.fsencode(path), C.byref(pv), C.byref(nv), C.byref(pf), C.byref(nf)))
    try:
        v = np.ctypeslib.as_array(pv, (max(1, nv.value) * 3,))[: 3 * nv.value].reshape(-1, 3).copy()
        f = np.ctypeslib.as_array(pf, (max(1, nf.value) * 3,))[: 3 * nf.value].reshape(-1, 3).copy()
    finally:
        lib.bzr_obj_free(C.cast(pv, C.c_void_p))
        lib.bzr_obj_free(C.cast(pf, C.c_void_p))
    return v, f


class Scene:
    """BlazertScene<double> on the GPU (blazert/scene.h:38-115)."""

    def __init__(self):
        self._lib = library()
        self._h = C.c_void_p()
        _check(self._lib.bzr_scene_create(C.byref(self._h)))
        self.committed = False

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.bzr_scene_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- persistent format (bzr_scene_serialize / bzr_scene_deserialize) ---------------------
    def to_bytes(self) -> bytes:
        """The committed scene in the persistent format (inputs, build options, trees)."""
        n = self._lib.bzr_scene_serialize(self._h, None, 0)
        if n < 0:
            _check(int(n))
        buf = (C.c_uint8 * n)()
        m = self._lib.bzr_scene_serialize(self._h, buf, n)
        if m < 0:
            _check(int(m))
        return bytes(buf)

    @classmethod
    def from_bytes(cls, data: bytes) -> "Scene":
        """A committed scene from the persistent format, without rebuilding its trees."""
        self = cls.__new__(cls)
        self._lib = library()
        self._h = C.c_void_p()
        buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
        _check(self._lib.bzr_scene_deserialize(C.byref(self._h), buf, len(data)))
        self.committed = True
        return self

    def save(self, path):
        _check(self._lib.bzr_scene_save(self._h, os.fsencode(path)))

    @classmethod
    def load(cls, path) -> "Scene":
        self = cls.__new__(cls)
        self._lib = library()
        self._h = C.c_void_p()
        _check(self._lib.bzr_scene_load(C.byref(self._h), os.fsencode(path)))
        self.committed = True
        return self

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- geometry ---------------------------------------------------------------------------
    def _add(self, rc, gid):
        if rc == ESTATE:
            return INVALID_ID
        _check(rc)
        return int(gid.value)

    def add_mesh(self, vertices, triangles):
        v = _f64(vertices, 3)
        f = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        gid = C.c_uint32()
        return self._add(self._lib.bzr_add_mesh(self._h, v.ctypes.data_as(_dp), v.shape[0],
                                                f.ctypes.data_as(_u32p), f.shape[0],
                                                C.byref(gid)), gid)

    def add_spheres(self, centers, radii):
        c, r = _f64(centers, 3), _f64(radii)
        if c.shape[0] != r.shape[0]:
            raise BlazertError(EINVAL, "centers and radii differ in length")
        gid = C.c_uint32()
        return self._add(self._lib.bzr_add_spheres(self._h, c.ctypes.data_as(_dp),
                                                   r.ctypes.data_as(_dp), r.shape[0],
                                                   C.byref(gid)), gid)

    def add_planes(self, centers, dxs, dys, rotations):
        c, dx, dy = _f64(centers, 3), _f64(dxs), _f64(dys)
        rot = _f64(rotations, 9)
        n = c.shape[0]
        if not (dx.shape[0] == dy.shape[0] == rot.shape[0] == n):
            raise BlazertError(EINVAL, "plane arrays differ in length")
        gid = C.c_uint32()
        return self._add(self._lib.bzr_add_planes(self._h, c.ctypes.data_as(_dp),
                                                  dx.ctypes.data_as(_dp), dy.ctypes.data_as(_dp),
                                                  rot.ctypes.data_as(_dp), n, C.byref(gid)), gid)

    def add_cylinders(self, centers, semi_axes_a, semi_axes_b, heights, rotations):
        c, a, b, h = _f64(centers, 3), _f64(semi_axes_a), _f64(semi_axes_b), _f64(heights)
        rot = _f64(rotations, 9)
        n = c.shape[0]
        if not (a.shape[0] == b.shape[0] == h.shape[0] == rot.shape[0] == n):
            raise BlazertError(EINVAL, "cylinder arrays differ in length")
        gid = C.c_uint32()
        return self._add(self._lib.bzr_add_cylinders(self._h, c.ctypes.data_as(_dp),
                                                     a.ctypes.data_as(_dp), b.ctypes.data_as(_dp),
                                                     h.ctypes.data_as(_dp), rot.ctypes.data_as(_dp),
                                                     n, C.byref(gid)), gid)

    def commit(self, build_options: Optional[BuildOptions] = None, gpu_build: Optional[bool] = None):
        """blazert/scene.h:91-115.  gpu_build: None builds kinds of 65,536 primitives or more
        on the GPU and smaller ones on the host; True / False forces the GPU / the host.  The
        trees are the same either way (bzr_commit_ex)."""
        o = build_options or BuildOptions()
        opts = _OptsC(o.min_leaf_primitives, o.max_tree_depth, o.bin_size)
        flags = 0 if gpu_build is None else (1 if gpu_build else 2)
        _check(self._lib.bzr_commit_ex(self._h, C.byref(opts), flags))
        self.committed = True
        return True

    def tree(self, kind):
        """Node arrays of one kind's BVH in the reference's node order (bzr_scene_tree):
        bmin, bmax (n x 3), leaf, axis, children (n x 2), prim_cnt, prim_ids."""
        k = ("mesh", "spheres", "planes", "cylinders").index(kind)
        f = self._lib.bzr_scene_tree
        n = f(self._h, k, None, None, None, None, None, None, None, 0)
        if n < 0:
            _check(int(n))
        bmin, bmax = np.zeros((n, 3)), np.zeros((n, 3))
        leaf, axis = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        ch, cnt = np.zeros((n, 2), np.uint32), np.zeros(n, np.uint32)
        f(self._h, k, bmin.ctypes.data, bmax.ctypes.data, leaf.ctypes.data, axis.ctypes.data,
          ch.ctypes.data, cnt.ctypes.data, None, 0)
        prims = np.zeros(max(int(cnt.sum()), 1), np.uint32)
        f(self._h, k, bmin.ctypes.data, bmax.ctypes.data, leaf.ctypes.data, axis.ctypes.data,
          ch.ctypes.data, cnt.ctypes.data, prims.ctypes.data, int(cnt.sum()))
        return dict(bmin=bmin, bmax=bmax, leaf=leaf, axis=axis, children=ch, prim_cnt=cnt,
                    prim_ids=prims[:int(cnt.sum())])

    def stats(self, kind):
        kinds = ("mesh", "spheres", "planes", "cylinders")
        n = C.c_uint64(); d = C.c_uint32(); s = C.c_double()
        _check(self._lib.bzr_scene_stats(self._h, kinds.index(kind), C.byref(n), C.byref(d),
                                         C.byref(s)))
        return dict(nodes=int(n.value), max_depth=int(d.value), build_seconds=float(s.value))

    # -- queries ----------------------------------------------------------------------------
    def intersect1(self, ray: Ray, rayhit: Optional[RayHit] = None):
        o, d = _f64(ray.origin), _f64(ray.direction)
        rh = _RayHitC()
        hit = C.c_int()
        _check(self._lib.bzr_intersect1_ex(self._h, o.ctypes.data_as(_dp), d.ctypes.data_as(_dp),
                                           float(ray.min_hit_distance),
                                           float(ray.max_hit_distance),
                                           RAY_ANY_HIT if ray.any_hit else 0, C.byref(rh),
                                           C.byref(hit)))
        if rayhit is None:
            rayhit = RayHit()
        if hit.value:  # on a miss the rayhit is left untouched, as in the reference
            rayhit.normal = np.array(rh.normal[:])
            rayhit.uv = np.array(rh.uv[:])
            rayhit.hit_distance = rh.hit_distance
            rayhit.prim_id = rh.prim_id
            rayhit.geom_id = rh.geom_id
        return bool(hit.value), rayhit

    def intersectN(self, origins, directions, tmin=None, tmax=None, mode="fp64", out=None,
                   stream=None, any_hit=False):
        """intersect1 over a batch.  numpy inputs: host path, returns numpy arrays when the
        results are in place.  torch CUDA tensors: device path, queued on ``stream`` (default:
        torch's current stream), returns torch tensors without waiting.  any_hit: every ray
        with Ray::AnyHit::yes."""
        flags = RAY_ANY_HIT if any_hit else 0
        try:
            import torch
            is_torch = isinstance(origins, torch.Tensor)
        except ImportError:
            is_torch = False
        if is_torch and origins.is_cuda:
            return self._intersect_device(origins, directions, tmin, tmax, mode, out, stream,
                                          flags)
        o, d = _f64(origins, 3), _f64(directions, 3)
        n = o.shape[0]
        tmn = None if tmin is None else np.ascontiguousarray(np.broadcast_to(tmin, (n,)), np.float64)
        tmx = None if tmax is None else np.ascontiguousarray(np.broadcast_to(tmax, (n,)), np.float64)
        if out is None:
            out = dict(t=np.empty(n), uv=np.empty((n, 2)), normal=np.empty((n, 3)),
                       prim=np.empty(n, np.uint32), geom=np.empty(n, np.uint32),
                       hit=np.empty(n, np.uint8))
        ptr = lambda a: None if a is None else a.ctypes.data
        _check(self._lib.bzr_intersectN_ex(self._h, n, ptr(o), ptr(d), ptr(tmn), ptr(tmx),
                                           ptr(out.get("t")), ptr(out.get("uv")),
                                           ptr(out.get("normal")), ptr(out.get("prim")),
                                           ptr(out.get("geom")), ptr(out.get("hit")),
                                           MODES[mode], flags, None))
        return out

    def _intersect_device(self, o, d, tmin, tmax, mode, out, stream, flags=0):
        import torch
        n = o.shape[0]
        dev = o.device
        f64 = torch.float64
        o = o.to(f64).contiguous()
        d = d.to(device=dev, dtype=f64).contiguous()
        tmn = None if tmin is None else torch.as_tensor(tmin, dtype=f64, device=dev).expand(n).contiguous()
        tmx = None if tmax is None else torch.as_tensor(tmax, dtype=f64, device=dev).expand(n).contiguous()
        if out is None:
            out = dict(t=torch.empty(n, dtype=f64, device=dev),
                       uv=torch.empty((n, 2), dtype=f64, device=dev),
                       normal=torch.empty((n, 3), dtype=f64, device=dev),
                       prim=torch.empty(n, dtype=torch.int32, device=dev),
                       geom=torch.empty(n, dtype=torch.int32, device=dev),
                       hit=torch.empty(n, dtype=torch.uint8, device=dev))
        st = (stream or torch.cuda.current_stream(dev)).cuda_stream
        ptr = lambda a: None if a is None else a.data_ptr()
        _check(self._lib.bzr_intersectN_ex(self._h, n, ptr(o), ptr(d), ptr(tmn), ptr(tmx),
                                           ptr(out.get("t")), ptr(out.get("uv")),
                                           ptr(out.get("normal")), ptr(out.get("prim")),
                                           ptr(out.get("geom")), ptr(out.get("hit")),
                                           MODES[mode], flags, C.c_void_p(st)))
        out["_keep"] = (o, d, tmn, tmx)
        return out

    def distance_to_surface(self, kind, prim_ids, points, closest=False, stream=None):
        """distance_to_surface of primitive prim_ids[i] of `kind` ("mesh", "spheres", "planes",
        "cylinders") and point i (bzr_distance_to_surface).  numpy inputs: returns numpy
        distances (and, for meshes with closest=True, the n x 3 closest points).  torch CUDA
        tensors: queued on ``stream`` (default: torch's current stream), returns tensors."""
        k = KIND_NAMES.index(kind)
        if closest and kind != "mesh":
            raise ValueError("closest points are returned for meshes only")
        if _is_cuda_tensor(points):
            import torch
            dev = points.device
            pts = points.to(torch.float64).contiguous()
            ids = torch.as_tensor(prim_ids, device=dev).to(torch.int32).contiguous()
            n = pts.shape[0]
            dist = torch.empty(n, dtype=torch.float64, device=dev)
            cl = torch.empty((n, 3), dtype=torch.float64, device=dev) if closest else None
            st = (stream or torch.cuda.current_stream(dev)).cuda_stream
            _check(self._lib.bzr_distance_to_surface(
                self._h, k, n, ids.data_ptr(), pts.data_ptr(), dist.data_ptr(),
                None if cl is None else cl.data_ptr(), C.c_void_p(st)))
            return (dist, cl) if closest else dist
        pts = _f64(points, 3)
        n = pts.shape[0]
        ids = np.ascontiguousarray(prim_ids, np.uint32).reshape(-1)
        if ids.shape[0] != n:
            raise ValueError("one primitive id per point")
        dist = np.empty(n)
        cl = np.empty((n, 3)) if closest else None
        _check(self._lib.bzr_distance_to_surface(self._h, k, n, ids.ctypes.data, pts.ctypes.data,
                                                 dist.ctypes.data,
                                                 None if cl is None else cl.ctypes.data, None))
        return (dist, cl) if closest else dist

    def closest_surface(self, points, stream=None):
        """Nearest surface of the scene per point (bzr_closest_surface): dict of distance,
        prim and geom (numpy for numpy input; torch tensors, queued on ``stream``, for CUDA
        tensors)."""
        if _is_cuda_tensor(points):
            import torch
            dev = points.device
            pts = points.to(torch.float64).contiguous()
            n = pts.shape[0]
            out = dict(distance=torch.empty(n, dtype=torch.float64, device=dev),
                       prim=torch.empty(n, dtype=torch.int32, device=dev),
                       geom=torch.empty(n, dtype=torch.int32, device=dev))
            st = (stream or torch.cuda.current_stream(dev)).cuda_stream
            _check(self._lib.bzr_closest_surface(self._h, n, pts.data_ptr(),
                                                 out["distance"].data_ptr(),
                                                 out["prim"].data_ptr(), out["geom"].data_ptr(),
                                                 C.c_void_p(st)))
            out["_keep"] = pts
            return out
        pts = _f64(points, 3)
        n = pts.shape[0]
        out = dict(distance=np.empty(n), prim=np.empty(n, np.uint32), geom=np.empty(n, np.uint32))
        _check(self._lib.bzr_closest_surface(self._h, n, pts.ctypes.data,
                                             out["distance"].ctypes.data,
                                             out["prim"].ctypes.data, out["geom"].ctypes.data,
                                             None))
        return out

    def tune(self, sort=None, sort_min_rays=None, threads=None, shared_stack=None, chunk=None,
             host_chunks=None, host_min_chunk=None, host_edge=None, host_grid_div=None,
             top_nodes=None):
        """Speed knobs (bzr_scene_tune); results do not depend on them.  sort: coherence sort
        of each batch; threads: 64 / 128 / 256 per block; shared_stack: traversal stack in
        shared memory instead of thread-local; chunk: rays per warp fetch (32 / 64 / 128, or 0
        for exactly the idle lanes); host_chunks / host_min_chunk: the pipeline of host-array
        calls (at most this many chunks, 1 to 32, of at least this many rays) and host_edge,
        the rays of an extra small first and last chunk (0: none); top_nodes: top-level nodes
        each block stages in shared memory (0 to 256)."""
        if top_nodes is not None:
            _check(self._lib.bzr_scene_tune(self._h, 10, int(top_nodes)))
        if host_grid_div is not None:
            _check(self._lib.bzr_scene_tune(self._h, 9, int(host_grid_div)))
        if host_edge is not None:
            _check(self._lib.bzr_scene_tune(self._h, 8, int(host_edge)))
        if host_chunks is not None:
            _check(self._lib.bzr_scene_tune(self._h, 6, int(host_chunks)))
        if host_min_chunk is not None:
            _check(self._lib.bzr_scene_tune(self._h, 7, int(host_min_chunk)))
        if sort is not None:
            _check(self._lib.bzr_scene_tune(self._h, 1, int(bool(sort))))
        if sort_min_rays is not None:
            _check(self._lib.bzr_scene_tune(self._h, 2, int(sort_min_rays)))
        if threads is not None:
            _check(self._lib.bzr_scene_tune(self._h, 3, int(threads)))
        if shared_stack is not None:
            _check(self._lib.bzr_scene_tune(self._h, 4, int(bool(shared_stack))))
        if chunk is not None:
            _check(self._lib.bzr_scene_tune(self._h, 5, int(chunk)))

    def build_statistics(self, kind):
        """The reference's BVHBuildStatistics of one kind's BVH as built at commit
        (bzr_scene_build_statistics): max_tree_depth, leaf_nodes, max_num_prims_per_leaf,
        min_num_prims_per_leaf, branch_nodes, bad_splits, build_seconds."""

        class _Stats(C.Structure):
            _fields_ = [(n, C.c_uint32) for n in ("max_tree_depth", "leaf_nodes",
                                                   "max_num_prims_per_leaf",
                                                   "min_num_prims_per_leaf", "branch_nodes",
                                                   "bad_splits")] + [("build_seconds", C.c_double)]

        st = _Stats()
        _check(self._lib.bzr_scene_build_statistics(self._h, KIND_NAMES.index(kind), C.byref(st)))
        return {n: getattr(st, n) for n, _ in _Stats._fields_}

    def work_counts(self, origins, directions, tmin=None, tmax=None, stream=None, mode="fp64"):
        """Box tests, primitive tests, node fetches and leaf fetches per kind for a batch in
        either mode (counting kernel; see bzr_work_counts_ex).  Returns dict(box=[4],
        prim=[4], node=[4], leaf=[4])."""
        tot = (C.c_uint64 * 16)()
        try:
            import torch
            dev = isinstance(origins, torch.Tensor) and origins.is_cuda
        except ImportError:
            dev = False
        if dev:
            import torch
            n = origins.shape[0]
            o = origins.to(torch.float64).contiguous()
            d = directions.to(torch.float64).contiguous()
            tmn = None if tmin is None else torch.as_tensor(tmin, dtype=torch.float64, device=o.device).expand(n).contiguous()
            tmx = None if tmax is None else torch.as_tensor(tmax, dtype=torch.float64, device=o.device).expand(n).contiguous()
            st = (stream or torch.cuda.current_stream(o.device)).cuda_stream
            ptr = lambda a: None if a is None else a.data_ptr()
            _check(self._lib.bzr_work_counts_ex(self._h, n, ptr(o), ptr(d), ptr(tmn), ptr(tmx),
                                                MODES[mode], tot, C.c_void_p(st)))
        else:
            o, d = _f64(origins, 3), _f64(directions, 3)
            n = o.shape[0]
            tmn = None if tmin is None else np.ascontiguousarray(np.broadcast_to(tmin, (n,)), np.float64)
            tmx = None if tmax is None else np.ascontiguousarray(np.broadcast_to(tmax, (n,)), np.float64)
            ptr = lambda a: None if a is None else a.ctypes.data
            _check(self._lib.bzr_work_counts_ex(self._h, n, ptr(o), ptr(d), ptr(tmn), ptr(tmx),
                                                MODES[mode], tot, None))
        return {k: [int(x) for x in tot[4 * j:4 * j + 4]]
                for j, k in enumerate(("box", "prim", "node", "leaf"))}

    def adjoint(self, origins, directions, fwd, grad_t=None, grad_uv=None, grad_normal=None,
                n_vertices=0, n_spheres=0, stream=None):
        """Gradients of the closest-hit outputs (bzr_adjoint_hit).  All tensors on the scene's
        CUDA device; fwd is the dict returned by intersectN.  Returns dict of gradients:
        origins, directions (n x 3), vertices (n_vertices x 3), centers (n_spheres x 3),
        radii (n_spheres)."""
        import torch

        dev = origins.device
        f64 = torch.float64
        n = origins.shape[0]
        g = dict(origins=torch.empty((n, 3), dtype=f64, device=dev),
                 directions=torch.empty((n, 3), dtype=f64, device=dev),
                 vertices=torch.empty((n_vertices, 3), dtype=f64, device=dev) if n_vertices else None,
                 centers=torch.empty((n_spheres, 3), dtype=f64, device=dev) if n_spheres else None,
                 radii=torch.empty(n_spheres, dtype=f64, device=dev) if n_spheres else None)
        ptr = lambda a: None if a is None else a.contiguous().data_ptr()
        keep = [origins.contiguous(), directions.contiguous()] + \
            [None if x is None else x.contiguous().to(f64) for x in (grad_t, grad_uv, grad_normal)]
        st = (stream or torch.cuda.current_stream(dev)).cuda_stream
        _check(self._lib.bzr_adjoint_hit(
            self._h, n, ptr(keep[0]), ptr(keep[1]), ptr(fwd["t"]), ptr(fwd["prim"]),
            ptr(fwd["geom"]), ptr(fwd["hit"]), ptr(keep[2]), ptr(keep[3]), ptr(keep[4]),
            ptr(g["vertices"]), ptr(g["centers"]), ptr(g["radii"]), ptr(g["origins"]),
            ptr(g["directions"]), C.c_void_p(st)))
        g["_keep"] = keep
        return g

    def check(self, stream=None, timeout_ms=60000):
        """Waits (bounded) for queued device work and raises if a kernel's bounds check fired."""
        flags = C.c_uint32()
        st = None if stream is None else C.c_void_p(stream)
        _check(self._lib.bzr_scene_check(self._h, st, int(timeout_ms), C.byref(flags)))
        return int(flags.value)


class Batch:
    """Many committed scenes traced together (bzr_batch_*), device arrays only."""

    def __init__(self, scenes):
        self._lib = library()
        self.scenes = list(scenes)  # keep the scenes alive
        arr = (C.c_void_p * len(self.scenes))(*[s._h.value for s in self.scenes])
        self._h = C.c_void_p()
        _check(self._lib.bzr_batch_create(C.byref(self._h), arr, len(self.scenes)))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.bzr_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tune(self, threads=None, shared_stack=None, stack_depth=None, sort=None,
             node_width=None):
        """Launch shape and ray order of the batch kernels (bzr_batch_tune): threads per block,
        stack storage, entries of the thread-local stack (32 or 64), the per-scene coherence
        sort and the node width of the mixed mode's walk (8 wide nodes or 2 binary nodes);
        results do not depend on them."""
        if threads is not None:
            _check(self._lib.bzr_batch_tune(self._h, 3, int(threads)))
        if shared_stack is not None:
            _check(self._lib.bzr_batch_tune(self._h, 4, int(bool(shared_stack))))
        if stack_depth is not None:
            _check(self._lib.bzr_batch_tune(self._h, 11, int(stack_depth)))
        if sort is not None:
            _check(self._lib.bzr_batch_tune(self._h, 1, int(bool(sort))))
        if node_width is not None:
            _check(self._lib.bzr_batch_tune(self._h, 12, int(node_width)))

    def intersect(self, ray_offsets, origins, directions, tmin=None, tmax=None, out=None,
                  timestamps=None, mode="fp64", stream=None):
        """ray_offsets: host sequence of n_scenes + 1 ints; rays: torch CUDA tensors (all
        scenes concatenated).  timestamps: optional int64 CUDA tensor of n_scenes + 1."""
        import torch

        n = origins.shape[0]
        dev = origins.device
        f64 = torch.float64
        if out is None:
            out = dict(t=torch.empty(n, dtype=f64, device=dev),
                       uv=torch.empty((n, 2), dtype=f64, device=dev),
                       normal=torch.empty((n, 3), dtype=f64, device=dev),
                       prim=torch.empty(n, dtype=torch.int32, device=dev),
                       geom=torch.empty(n, dtype=torch.int32, device=dev),
                       hit=torch.empty(n, dtype=torch.uint8, device=dev))
        offs = (C.c_uint64 * len(ray_offsets))(*[int(x) for x in ray_offsets])
        ptr = lambda a: None if a is None else a.data_ptr()
        st = (stream or torch.cuda.current_stream(dev)).cuda_stream
        _check(self._lib.bzr_batch_intersect(
            self._h, offs, ptr(origins), ptr(directions), ptr(tmin), ptr(tmax), ptr(out.get("t")),
            ptr(out.get("uv")), ptr(out.get("normal")), ptr(out.get("prim")), ptr(out.get("geom")),
            ptr(out.get("hit")), ptr(timestamps), MODES[mode], C.c_void_p(st)))
        return out

    def check(self, stream=None):
        flags = C.c_uint32()
        _check(self._lib.bzr_batch_check(self._h, None if stream is None else C.c_void_p(stream),
                                         C.byref(flags)))
        return int(flags.value)


def intersect1(scene: Scene, ray: Ray, rayhit: RayHit) -> bool:
    """blazert/scene.h:161-162: fills rayhit on a hit and returns whether anything was hit."""
    hit, _ = scene.intersect1(ray, rayhit)
    return hit


__all__ = ["Scene", "Batch", "Ray", "RayHit", "BuildOptions", "intersect1", "BlazertError", "INVALID_ID",
           "DBL_MAX", "RAY_ANY_HIT", "library"]
