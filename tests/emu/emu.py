"""ctypes loader for the CPU emulator of the GPU traversal (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from oracle.oracle import (_Base, _CREATE_ARGS, _DIST_ARGS, _NEAREST_ARGS, _TREE_ARGS,
                           _closest_surface, _distance_to_surface, _dp, _outputs, _ptr, _rays,
                           _u32p, _u8p)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libbzr_emu.so")
KINDS = ("mesh", "spheres", "planes", "cylinders")
_lib = None


def build(force=False, out=None, flags=()):
    """Compiles the emulator with the host compiler (no GPU or nvcc needed); `out` and `flags`
    build a variant elsewhere (the sanitizer run)."""
    root = os.path.dirname(os.path.dirname(HERE))
    srcs = [os.path.join(HERE, "emu.cpp"), os.path.join(root, "blazert_b200", "csrc", "scene.cpp"),
            os.path.join(root, "blazert_b200", "csrc", "scene_io.cpp"),
            os.path.join(root, "blazert_b200", "csrc", "obj.cpp")]
    if out is not None:
        cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
        subprocess.run([os.environ.get("BZR_CXX", "g++"), "-std=c++17", "-O1", "-g",
                        "-ffp-contract=off", "-fPIC", "-fopenmp", "-shared", "-I", cuda_inc,
                        *flags] + srcs + ["-o", out], check=True)
        return out
    deps = srcs + [os.path.join(root, "blazert_b200", "csrc", f)
                   for f in ("layout.h", "scene.h", "trace_core.cuh", "distance_core.cuh")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in deps):
        return LIB
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run([os.environ.get("BZR_CXX", "g++"), "-std=c++17", "-O2", "-ffp-contract=off",
                    "-fPIC", "-fopenmp", "-shared", "-I", cuda_inc] + srcs + ["-o", LIB], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        lib = C.CDLL(build())
        lib.emu_scene_create.restype = C.c_void_p
        lib.emu_scene_create.argtypes = _CREATE_ARGS
        lib.emu_scene_destroy.argtypes = [C.c_void_p]
        lib.emu_scene_tree.restype = C.c_long
        lib.emu_scene_tree.argtypes = _TREE_ARGS
        lib.emu_scene_intersect.restype = C.c_uint32
        lib.emu_scene_intersect.argtypes = [C.c_void_p, C.c_long, _dp, _dp, _dp, _dp, _dp, _dp,
                                            _dp, _u32p, _u32p, _u8p, C.c_uint32, C.c_int]
        lib.emu_prim_box.argtypes = [C.c_void_p, C.c_int, C.c_uint32, _dp, _dp, _dp]
        lib.emu_box_accept.argtypes = [_dp, _dp, _dp, _dp, C.c_double, C.c_double]
        lib.emu_build_statistics.argtypes = [C.c_void_p, C.c_int, _u32p]
        lib.emu_image_digest.argtypes = [C.c_void_p, C.c_int, C.c_long, C.c_void_p]
        lib.emu_scene_encode.restype = C.c_long
        lib.emu_scene_encode.argtypes = [C.c_void_p, C.c_void_p, C.c_long]
        lib.emu_scene_decode.restype = C.c_void_p
        lib.emu_scene_decode.argtypes = [C.c_void_p, C.c_long, C.c_char_p, C.c_long]
        lib.emu_distance_to_surface.restype = C.c_uint32
        lib.emu_distance_to_surface.argtypes = _DIST_ARGS
        lib.emu_closest_surface.argtypes = _NEAREST_ARGS
        lib.emu_work_counts.argtypes = [C.c_void_p, C.c_long, _dp, _dp, _dp, _dp, C.c_int,
                                        C.c_void_p]
        lib.emu_wide_check.restype = C.c_long
        lib.emu_wide_check.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_long)]
        _lib = lib
    return _lib


def box_accept(bmin, bmax, org, direction, tmin, tmax):
    """Decision of the kernels' deferred slab test for one box at hit distance tmax."""
    f = lambda a: np.ascontiguousarray(a, np.float64)
    return bool(load().emu_box_accept(_ptr(f(bmin), _dp), _ptr(f(bmax), _dp), _ptr(f(org), _dp),
                                      _ptr(f(direction), _dp), float(tmin), float(tmax)))


class EmuScene(_Base):
    _prefix = "emu_"

    def __init__(self, spec, **kw):
        self._lib = load()
        super().__init__(spec, **kw)

    def prim_box(self, kind, prim_id):
        mn, mx, c = np.zeros(3), np.zeros(3), np.zeros(3)
        rc = self._lib.emu_prim_box(self._h, KINDS.index(kind), prim_id, _ptr(mn, _dp),
                                    _ptr(mx, _dp), _ptr(c, _dp))
        assert rc == 0
        return mn, mx, c

    def build_statistics(self, kind):
        """The host builder's statistics of one kind (tree_statistics in scene.cpp)."""
        import numpy as np
        from oracle.oracle import STAT_KEYS

        out = np.zeros(6, np.uint32)
        if self._lib.emu_build_statistics(self._h, KINDS.index(kind), _ptr(out, _u32p)) != 0:
            return None
        return dict(zip(STAT_KEYS, (int(x) for x in out)))

    def image_digest(self, kind, workers):
        """Digest of one kind's device image flattened with at most `workers` threads."""
        out = np.zeros(1, np.uint64)
        if self._lib.emu_image_digest(self._h, KINDS.index(kind), workers, out.ctypes.data) != 0:
            return None
        return int(out[0])

    def encode(self) -> bytes:
        """The scene in the persistent format (scene_io.cpp)."""
        n = self._lib.emu_scene_encode(self._h, None, 0)
        buf = (C.c_uint8 * n)()
        self._lib.emu_scene_encode(self._h, buf, n)
        return bytes(buf)

    @classmethod
    def decode(cls, data: bytes) -> "EmuScene":
        """A scene from the persistent format; ValueError with the reason when refused."""
        self = cls.__new__(cls)
        self._lib = load()
        why = C.create_string_buffer(256)
        buf = (C.c_uint8 * max(1, len(data))).from_buffer_copy(data or b"\0")
        h = self._lib.emu_scene_decode(buf, len(data), why, 256)
        if not h:
            raise ValueError(why.value.decode())
        self._h = h
        self._keep = None
        self.geom_ids = {}
        return self

    def distance_to_surface(self, kind, ids, points):
        """The distance kernel's per-point code on the CPU."""
        return _distance_to_surface(self, kind, ids, points)

    def closest_surface(self, points):
        """The nearest-surface kernel's per-point code (BVH pruning included) on the CPU."""
        return _closest_surface(self, points)

    def intersect(self, org, dirs, tmin=None, tmax=None, stack_cap=0, mode="fp64", any_hit=False):
        """mode fp64 | mixed; any_hit: every ray with Ray::AnyHit::yes."""
        org, dirs, tmin, tmax, n = _rays(org, dirs, tmin, tmax)
        out = _outputs(n)
        out["error_word"] = int(self._lib.emu_scene_intersect(
            self._h, n, _ptr(org, _dp), _ptr(dirs, _dp), _ptr(tmin, _dp), _ptr(tmax, _dp),
            _ptr(out["t"], _dp), _ptr(out["uv"], _dp), _ptr(out["normal"], _dp),
            _ptr(out["prim"], _u32p), _ptr(out["geom"], _u32p), _ptr(out["hit"], _u8p), stack_cap,
            (1 if mode == "mixed" else 0) | (2 if any_hit else 0)))
        return out

    def work_counts(self, org, dirs, tmin=None, tmax=None, mode="fp64"):
        """The kernels' work counters over a batch: dict of box, prim, node, leaf (4 per kind)."""
        org, dirs, tmin, tmax, n = _rays(org, dirs, tmin, tmax)
        tot = np.zeros(16, np.uint64)
        self._lib.emu_work_counts(self._h, n, _ptr(org, _dp), _ptr(dirs, _dp), _ptr(tmin, _dp),
                                  _ptr(tmax, _dp), 1 if mode == "mixed" else 0, tot.ctypes.data)
        return {k: [int(x) for x in tot[4 * j:4 * j + 4]]
                for j, k in enumerate(("box", "prim", "node", "leaf"))}

    def wide_check(self, kind):
        """(violations, leaf records reached) of the kind's wide image, or None without one."""
        leaves = C.c_long(0)
        bad = self._lib.emu_wide_check(self._h, KINDS.index(kind), C.byref(leaves))
        return None if bad < 0 else (int(bad), int(leaves.value))
