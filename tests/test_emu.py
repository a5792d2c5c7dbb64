"""The GPU kernels' per-ray code (blazert_b200/csrc/trace_core.cuh), compiled as host code by
the test-only emulator, against the CPU oracle: checks the device layout, the deferred-key
traversal and the primitive tests without a GPU."""
import numpy as np
import pytest

from blazert_b200 import workloads as W
from oracle.oracle import Oracle
from tests.emu.emu import EmuScene
from tests.helpers import mismatches
from tests.scenes import edge_case_scenes


MODES = ["fp64", "mixed"]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", ["icosphere_pinhole", "mixed_primitives", "heightfield"])
def test_workloads(name, mode):
    if name == "mixed_primitives":
        wl = W.mixed_primitives(n_rays=100_000)
    elif name == "heightfield":
        wl = W.heightfield(n_rays=50_000, grid=256)
    else:
        wl = W.WORKLOADS[name]()
    R = wl.rays
    ref = Oracle(wl.scene).intersect(R.origins, R.directions, R.tmin, R.tmax)
    got = EmuScene(wl.scene).intersect(R.origins, R.directions, R.tmin, R.tmax, mode=mode)
    assert got["error_word"] == 0
    assert mismatches(got, ref) == []


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", ["icosphere_pinhole", "mixed_primitives", "heightfield"])
def test_any_hit(name, mode):
    """Rays with Ray::AnyHit::yes: the kernels' leaf step ends the traversal at the first hit,
    as the oracle (pinned to the reference) does."""
    if name == "mixed_primitives":
        wl = W.mixed_primitives(n_rays=100_000)
    elif name == "heightfield":
        wl = W.heightfield(n_rays=50_000, grid=256)
    else:
        wl = W.WORKLOADS[name]()
    R = wl.rays
    ref = Oracle(wl.scene).intersect(R.origins, R.directions, R.tmin, R.tmax, any_hit=True)
    closest = Oracle(wl.scene).intersect(R.origins, R.directions, R.tmin, R.tmax)
    assert (ref["prim"] != closest["prim"]).any()  # the flag changes which hit is reported
    got = EmuScene(wl.scene).intersect(R.origins, R.directions, R.tmin, R.tmax, mode=mode,
                                       any_hit=True)
    assert got["error_word"] == 0
    assert mismatches(got, ref) == []


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("case", edge_case_scenes(), ids=lambda c: c[0])
def test_edge_cases(case, mode):
    _, spec, R = case
    ref = Oracle(spec).intersect(R.origins, R.directions, R.tmin, R.tmax)
    got = EmuScene(spec).intersect(R.origins, R.directions, R.tmin, R.tmax, mode=mode)
    assert got["error_word"] == 0
    assert mismatches(got, ref) == []


def test_build_options():
    wl = W.mixed_primitives(n_rays=20_000, n_spheres=3000, n_cylinders=300, n_planes=50, seed=9)
    R = wl.rays
    for opts in (dict(min_leaf=1, max_depth=28, bins=64), dict(min_leaf=8, max_depth=6, bins=16),
                 dict(min_leaf=2, max_depth=40, bins=3)):
        ref = Oracle(wl.scene, **opts).intersect(R.origins, R.directions)
        for mode in MODES:
            got = EmuScene(wl.scene, **opts).intersect(R.origins, R.directions, mode=mode)
            assert got["error_word"] == 0
            assert mismatches(got, ref) == [], (opts, mode)


def test_stack_overflow_is_flagged_not_silent():
    """A stack too small for the tree sets the error word and the ray stops; it never writes
    outside the stack (the GPU kernels run the same code)."""
    wl = W.icosphere_pinhole(level=4, width=64, height=64)
    R = wl.rays
    got = EmuScene(wl.scene).intersect(R.origins, R.directions, stack_cap=1)
    assert got["error_word"] & 1


def test_flatten_image_does_not_depend_on_threads():
    """The flattener runs its long loops (node fill, leaf-ordered primitives, vertex numbering
    by first use) over ranges on several threads.  The device image must be the same bytes for
    every thread count; the sizes make each loop split into several ranges."""
    rng = np.random.default_rng(11)
    n = 200_000
    spec = W.SceneSpec().add_mesh(*W.icosphere(7)).add_spheres(
        rng.uniform(-10.0, 10.0, (n, 3)), rng.uniform(0.01, 0.1, n))
    emu = EmuScene(spec)
    for kind in ("mesh", "spheres"):
        one = emu.image_digest(kind, 1)
        assert [emu.image_digest(kind, w) for w in (2, 3, 16)] == [one] * 3, kind
    assert emu.image_digest("planes", 4) is None


POISON_RUN = r'''
import hashlib, json, os, sys
import numpy as np
sys.path.insert(0, os.environ["BZR_ROOT"])
import tests.emu.emu as E
E.build = lambda force=False, out=None, flags=(): os.environ["BZR_EMU_LIB"]
from tests.test_emu import _raw_storage_results
print(json.dumps(_raw_storage_results()))
'''


def _raw_storage_results():
    """Image digests (every kind, 1 and 16 threads) and scene-file hashes of scenes that take
    the threaded paths, small and edge-case scenes."""
    rng = np.random.default_rng(12)
    n = 150_000
    specs = [W.SceneSpec().add_mesh(*W.icosphere(7)).add_spheres(
                 rng.uniform(-10.0, 10.0, (n, 3)), rng.uniform(0.01, 0.1, n)),
             W.mixed_primitives(n_rays=16).scene]
    specs += [spec for _, spec, _ in edge_case_scenes()]
    out = []
    for spec in specs:
        emu = EmuScene(spec)
        out.append([emu.image_digest(k, w) for k in spec.order for w in (1, 16)])
        data = emu.encode()
        out.append(__import__("hashlib").sha256(data).hexdigest())
        out.append(EmuScene.decode(data).encode() == data)
    return out


def test_raw_storage_is_written_in_full(tmp_path):
    """The host arrays allocated without zero-fill (prim boxes, tree nodes, device images, the
    scene-file buffer) must be written in full: an emulator built with BZR_POISON_RAW, which
    fills that storage with 0xA5 bytes when it is allocated, gives the same images and files as
    the normal build."""
    import json
    import os
    import subprocess
    import sys

    from tests.emu import emu as E

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib = E.build(out=str(tmp_path / "libemu_poison.so"), flags=("-DBZR_POISON_RAW",))
    script = tmp_path / "run.py"
    script.write_text(POISON_RUN)
    r = subprocess.run([sys.executable, str(script)], capture_output=True, text=True, timeout=900,
                       env=dict(os.environ, BZR_EMU_LIB=lib, BZR_ROOT=root))
    assert r.returncode == 0, r.stderr[-3000:]
    poisoned = json.loads(r.stdout.strip().splitlines()[-1])
    assert poisoned == json.loads(json.dumps(_raw_storage_results()))


@pytest.mark.parametrize("name", ["icosphere_pinhole", "mixed_primitives", "heightfield"])
def test_wide_image_contains_every_leaf(name):
    """The mixed path's wide image: every leaf record is reached once from the wide root, each
    quantised child box on the way contains the leaf's exact box, and the records hold the
    tree leaves' exact boxes and primitive ranges.  Cylinders have no wide image (their hit
    distance may grow, so their mixed mode runs the FP64 traversal)."""
    kw = {"n_rays": 16}
    if name == "heightfield":
        kw["grid"] = 256
    wl = W.WORKLOADS[name](**kw)
    emu = EmuScene(wl.scene)
    for kind in wl.scene.order:
        got = emu.wide_check(kind)
        if kind == "cylinders":
            assert got is None
            continue
        bad, leaves = got
        assert bad == 0 and leaves == emu.build_statistics(kind)["leaf_nodes"], (kind, got)


def test_mixed_walk_uses_the_wide_image():
    """The mixed path fetches far fewer nodes than the FP64 path on the same rays (wide nodes
    of up to 8 children) and tests the same primitives."""
    wl = W.heightfield(n_rays=20_000, grid=256)
    R = wl.rays
    emu = EmuScene(wl.scene)
    a = emu.work_counts(R.origins, R.directions, R.tmin, R.tmax, mode="fp64")
    b = emu.work_counts(R.origins, R.directions, R.tmin, R.tmax, mode="mixed")
    assert a["prim"] == b["prim"]
    assert b["node"][0] * 2 < a["node"][0]
    assert b["leaf"][0] >= a["leaf"][0]


def _grazing_rays(spec, n, rng):
    """Rays aimed at box faces, edges and corners of the scene's primitives: origins on a face
    plane or a corner, directions along an axis with tiny or zero other components, finite
    tmax ending inside boxes, tmin > 0 starting inside them."""
    emu = EmuScene(spec)
    boxes = []
    for kind in spec.order:
        m = len(next(iter(getattr(spec, kind).values()))) if kind != "mesh" else \
            len(spec.mesh["faces"])
        for pid in rng.integers(0, m, min(m, 64)):
            boxes.append(emu.prim_box(kind, int(pid))[:2])
    org, dirs, tmin, tmax = [], [], [], []
    for _ in range(n):
        lo, hi = boxes[rng.integers(len(boxes))]
        p = np.where(rng.random(3) < 0.5, lo, hi)
        if rng.random() < 0.5:  # a point on a face instead of a corner
            a = rng.integers(3)
            p = p.copy()
            p[a] = rng.uniform(lo[a], hi[a])
        d = np.zeros(3)
        a = rng.integers(3)
        d[a] = rng.choice([-1.0, 1.0])
        small = rng.choice([0.0, 1e-30, 1e-12, 1e-6, 1e-3])
        d[(a + 1) % 3] = small * rng.choice([-1.0, 1.0])
        d[(a + 2) % 3] = rng.choice([0.0, small, -small])
        back = rng.uniform(0.0, 5.0)
        org.append(p - back * d)
        dirs.append(d * rng.choice([1.0, 3.0, 1e-3]))
        tmin.append(rng.choice([0.0, 0.0, back * 0.5, back]))
        tmax.append(rng.choice([np.inf, 1.7976931348623157e308, back + rng.uniform(0, 2)]))
    return (np.array(org), np.array(dirs), np.array(tmin), np.array(tmax))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_mixed_grazing_rays_match_the_oracle(seed):
    """Rays that graze box faces, edges and corners, run parallel to slab planes or start and
    end inside boxes: the mixed path's FP32 walk with the exact FP64 leaf test gives the
    oracle's results bit for bit (rays with a zero direction component take the FP64 walk)."""
    rng = np.random.default_rng(100 + seed)
    specs = [W.icosphere_pinhole(level=3, width=8, height=8).scene,
             W.mixed_primitives(n_rays=16, n_spheres=500, n_cylinders=50, n_planes=40,
                                seed=seed).scene,
             W.heightfield(n_rays=16, grid=64).scene]
    for spec in specs:
        o, d, tmn, tmx = _grazing_rays(spec, 4000, rng)
        ref = Oracle(spec).intersect(o, d, tmn, tmx)
        got = EmuScene(spec).intersect(o, d, tmn, tmx, mode="mixed")
        assert got["error_word"] == 0
        assert mismatches(got, ref) == []
