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
