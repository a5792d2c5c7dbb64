"""ctypes loader for the CPU emulator of the GPU traversal (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from oracle.oracle import _Base, _CREATE_ARGS, _TREE_ARGS, _dp, _outputs, _ptr, _rays, _u32p, _u8p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libbzr_emu.so")


def build(force=False):
    """Compiles the emulator with the host compiler (no GPU or nvcc needed)."""
    import subprocess
    root = os.path.dirname(os.path.dirname(HERE))
    srcs = [os.path.join(HERE, "emu.cpp"), os.path.join(root, "blazert_b200", "csrc", "scene.cpp")]
    deps = srcs + [os.path.join(root, "blazert_b200", "csrc", f)
                   for f in ("layout.h", "scene.h", "trace_core.cuh")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in deps):
        return LIB
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run([os.environ.get("BZR_CXX", "g++"), "-std=c++17", "-O2", "-ffp-contract=off",
                    "-fPIC", "-fopenmp", "-shared", "-I", cuda_inc] + srcs + ["-o", LIB], check=True)
    return LIB


class EmuScene(_Base):
    _prefix = "emu_"
    _lib = None

    def __init__(self, spec, **kw):
        if EmuScene._lib is None:
            lib = C.CDLL(build())
            lib.emu_scene_create.restype = C.c_void_p
            lib.emu_scene_create.argtypes = _CREATE_ARGS
            lib.emu_scene_destroy.argtypes = [C.c_void_p]
            lib.emu_scene_tree.restype = C.c_long
            lib.emu_scene_tree.argtypes = _TREE_ARGS
            lib.emu_scene_intersect.restype = C.c_uint32
            lib.emu_scene_intersect.argtypes = [C.c_void_p, C.c_long, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                          _u32p, _u32p, _u8p, C.c_uint32]
            EmuScene._lib = lib
        super().__init__(spec, **kw)

    def intersect(self, org, dirs, tmin=None, tmax=None, stack_cap=0):
        org, dirs, tmin, tmax, n = _rays(org, dirs, tmin, tmax)
        out = _outputs(n)
        out["error_word"] = int(self._lib.emu_scene_intersect(
            self._h, n, _ptr(org, _dp), _ptr(dirs, _dp), _ptr(tmin, _dp), _ptr(tmax, _dp),
            _ptr(out["t"], _dp), _ptr(out["uv"], _dp), _ptr(out["normal"], _dp),
            _ptr(out["prim"], _u32p), _ptr(out["geom"], _u32p), _ptr(out["hit"], _u8p), stack_cap))
        return out
