"""The host code the product shares with the CPU emulator under AddressSanitizer and
UndefinedBehaviorSanitizer: scene.cpp (collections and their precompute, the binned-SAH
builder, flattening), scene_io.cpp (the scene file) and obj.cpp (the OBJ reader), plus the
kernels' per-ray and per-point code compiled for the CPU.  A child process with the sanitizer
runtime preloaded builds scenes (workloads and edge cases), traces rays, runs distance and
nearest-surface queries, writes and reads scene files (valid, damaged and fuzzed) and reads OBJ
files (valid and fuzzed).  Any report fails the test."""
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RUN = r'''
import ctypes as C
import os
import struct
import sys

import numpy as np

sys.path.insert(0, os.environ["BZR_ROOT"])
import tests.emu.emu as E

E.build = lambda force=False, out=None, flags=(): os.environ["BZR_EMU_LIB"]
from blazert_b200 import workloads as W
from tests.emu.emu import EmuScene
from tests.scenes import distance_queries, edge_case_scenes


def fnv1a(b):
    h = 1469598103934665603
    for x in b:
        h = ((h ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def reseal(body):
    """body followed by the hash its version field names (1: FNV-1a over the whole body; else
    FNV-1a over the FNV-1a hashes of its 2^20-byte blocks)."""
    if len(body) >= 12 and struct.unpack_from("<I", body, 8)[0] == 1:
        return body + struct.pack("<Q", fnv1a(body))
    blocks = b"".join(struct.pack("<Q", fnv1a(body[i:i + (1 << 20)]))
                      for i in range(0, len(body), 1 << 20))
    return body + struct.pack("<Q", fnv1a(blocks))


rng = np.random.default_rng(0)
scenes = [W.mixed_primitives(n_rays=2000, n_spheres=300, n_cylinders=60, n_planes=20, seed=3),
          W.icosphere_pinhole(n_rays=2000)]
scenes += [W.Workload(n, s, R, {}) for n, s, R in edge_case_scenes()]
for wl in scenes:
    spec, R = wl.scene, wl.rays
    for kw in (dict(), dict(min_leaf=1, max_depth=40, bins=3)):
        s = EmuScene(spec, **kw)
        m = min(R.n, 1500)
        for mode in ("fp64", "mixed"):
            out = s.intersect(R.origins[:m], R.directions[:m], None if R.tmin is None else R.tmin[:m],
                              None if R.tmax is None else R.tmax[:m], mode=mode)
            assert out["error_word"] == 0
        for kind in spec.order:
            ids, pts = distance_queries(spec, kind, rng, 300)
            s.distance_to_surface(kind, ids, pts)
        s.closest_surface(rng.uniform(-50, 50, (200, 3)))
        data = s.encode()
        assert EmuScene.decode(data).encode() == data
        body = data[:-8]
        for _ in range(40):
            b = bytearray(body)
            op = rng.integers(3)
            if op == 0:
                b[int(rng.integers(len(b)))] = int(rng.integers(256))
            elif op == 1:
                at = int(rng.integers(len(b)))
                b[at:at] = bytes(rng.integers(0, 256, 7, dtype=np.uint8))
            else:
                del b[int(rng.integers(len(b))):]
            try:
                t = EmuScene.decode(reseal(bytes(b)))
                t.intersect(R.origins[:64], R.directions[:64])
            except ValueError:
                pass

lib = C.CDLL(os.environ["BZR_EMU_LIB"])
lib.emu_obj_load.argtypes = [C.c_char_p, C.c_void_p, C.c_long, C.c_void_p, C.c_long,
                             C.POINTER(C.c_long), C.POINTER(C.c_long), C.c_char_p, C.c_long]
base = ("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 1e3\nvt 0 0\nvn 0 0 1\ng a\nf 1 2 3\n"
        "f 1/1/1 2/1/1 3/1/1 4/1\no b\nf -1 -2 -3 -4\nf 1//1 3//1 4//1\n")
path = os.path.join(os.environ["BZR_TMP"], "f.obj").encode()
nv, nf = C.c_long(), C.c_long()
why = C.create_string_buffer(256)
alphabet = b"0123456789 -+./eEvfgotn#\t\r\n"
for k in range(300):
    b = bytearray(base.encode())
    for _ in range(int(rng.integers(0, 6))):
        at = int(rng.integers(len(b)))
        ch = alphabet[int(rng.integers(len(alphabet)))]
        if rng.random() < 0.5:
            b[at] = ch
        else:
            b[at:at] = bytes([ch]) * int(rng.integers(1, 12))
    open(path, "wb").write(bytes(b))
    if lib.emu_obj_load(path, None, 0, None, 0, C.byref(nv), C.byref(nf), why, 256) == 0:
        v = np.empty(3 * nv.value + 1)
        f = np.empty(3 * nf.value + 1, np.uint32)
        assert lib.emu_obj_load(path, v.ctypes.data, v.size, f.ctypes.data, f.size, C.byref(nv),
                                C.byref(nf), why, 256) == 0
print("sanitized run ok")
'''


def _runtime(name):
    p = subprocess.run([os.environ.get("BZR_CC", "gcc"), f"-print-file-name={name}"],
                       capture_output=True, text=True).stdout.strip()
    return p if os.path.isabs(p) and os.path.exists(p) else None


@pytest.mark.skipif(_runtime("libasan.so") is None or shutil.which("g++") is None,
                    reason="no ASan runtime in this toolchain")
def test_host_code_under_asan_and_ubsan(tmp_path):
    from tests.emu import emu

    lib = emu.build(out=str(tmp_path / "libemu_san.so"),
                    flags=("-fsanitize=address,undefined", "-fno-omit-frame-pointer",
                           "-fno-sanitize-recover=undefined"))
    script = tmp_path / "run.py"
    script.write_text(RUN)
    env = dict(os.environ, LD_PRELOAD=_runtime("libasan.so"), BZR_EMU_LIB=lib, BZR_ROOT=ROOT,
               BZR_TMP=str(tmp_path), ASAN_OPTIONS="detect_leaks=0:abort_on_error=1",
               UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1", OMP_NUM_THREADS="2")
    r = subprocess.run([sys.executable, str(script)], env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0 and "sanitized run ok" in r.stdout, r.stderr[-4000:]
