"""Builds libblazert_b200.so in-tree (blazert_b200/_lib/) for sm_100a.

    python -m blazert_b200.build [--force] [--verbose]

trace.cu is compiled by nvcc for sm_100a only, with --fmad=false so that no multiply-add is
contracted (the kernels must reproduce the reference's double-precision results bit for bit);
the host sources are compiled with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libblazert_b200.so")
# measurement-only read-bandwidth probe (the roofline's L2 ceiling), kept out of the product
PROBE = os.path.join(LIBDIR, "libbzr_probe.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXX = os.environ.get("BZR_CXX", "g++")
HOST_FLAGS = ["-std=c++17", "-O3", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra"]
CU_FLAGS = ARCH + ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler",
                   "-fPIC,-ffp-contract=off", "-ccbin", CXX]

SOURCES = [("scene.cpp", "cxx"), ("capi.cpp", "cxx"), ("trace.cu", "cu"), ("adjoint.cu", "cu"),
           ("noalloc.cu", "cu"), ("batch.cpp", "cxx"), ("gbuild.cu", "cu"), ("distance.cu", "cu"),
           ("scene_io.cpp", "cxx"), ("obj.cpp", "cxx")]
HEADERS = ["layout.h", "scene.h", "trace.h", "trace_core.cuh", "adjoint.h", "capi_internal.h",
           "distance.h", "distance_core.cuh", "bucket_sort.cuh", "alloc.h"]


def _cuda_home():
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and os.path.exists(os.path.join(c, "bin", "nvcc")):
            return c
    nvcc = shutil.which("nvcc")
    if nvcc:
        return os.path.dirname(os.path.dirname(nvcc))
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_verbose=False):
    cuda = _cuda_home()
    nvcc = os.path.join(cuda, "bin", "nvcc")
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "blazert_b200.h")]
    objs = []
    for src, kind in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if not force and not _stale(o, [s] + hdrs):
            continue
        if kind == "cxx":
            cmd = [CXX] + HOST_FLAGS + ["-I", os.path.join(cuda, "include"), "-c", s, "-o", o]
        else:
            cmd = [nvcc] + CU_FLAGS + (["-Xptxas", "-v"] if ptxas_verbose else []) + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-ccbin", CXX, "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    probe_src = os.path.join(CSRC, "probe.cu")
    if force or _stale(PROBE, [probe_src]):
        cmd = [nvcc] + CU_FLAGS + ["-shared", "-o", PROBE, probe_src]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose, a.ptxas_verbose))


if __name__ == "__main__":
    sys.exit(main())
