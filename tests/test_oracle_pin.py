"""Pins the CPU oracle (oracle/bzr_oracle.c) to the reference itself.

oracle/_ref/libref_parity.so is the reference's own headers (blazert/scene.h and everything it
includes, unmodified) compiled against the blaze-API shim with -ffp-contract=off.  The oracle
must reproduce its BVHs node for node and its intersect1 results bit for bit.  The product's
host builder (via the emulator library) must reproduce the same trees."""
import numpy as np
import pytest

from blazert_b200 import workloads as W
from oracle.oracle import Oracle, RefScene
from tests.emu.emu import EmuScene
from tests.helpers import mismatches
from tests.scenes import edge_case_scenes

needs_ref = pytest.mark.skipif(not RefScene.available("parity"),
                               reason="oracle/_ref not built (reference sources absent)")


def same_tree(a, b):
    for key in a:
        x, y = a[key], b[key]
        if x.shape != y.shape:
            return f"{key}: shape {x.shape} vs {y.shape}"
        if x.dtype == np.float64:
            x, y = x.view(np.uint64), y.view(np.uint64)
        if not np.array_equal(x, y):
            return f"{key}: {int(np.count_nonzero(x != y))} entries differ"
    return None


def _cases():
    out = [("icosphere_pinhole", W.icosphere_pinhole().scene, W.icosphere_pinhole().rays)]
    wl = W.mixed_primitives(n_rays=100_000)
    out.append(("mixed_primitives", wl.scene, wl.rays))
    out += edge_case_scenes()
    return out


@needs_ref
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_oracle_matches_reference(case):
    _, spec, R = case
    ref = RefScene(spec)
    ora = Oracle(spec)
    assert ora.geom_ids == ref.geom_ids
    for kind in spec.order:
        assert same_tree(ora.tree(kind), ref.tree(kind)) is None, kind
    a = ora.intersect(R.origins, R.directions, R.tmin, R.tmax)
    b = ref.intersect(R.origins, R.directions, R.tmin, R.tmax)
    assert mismatches(a, b) == []


@needs_ref
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_oracle_any_hit_matches_reference(case):
    """Rays built with Ray::AnyHit::yes: each kind's traversal stops at the first leaf hit it
    accepts (blazert/bvh/intersect.h:73-75, accel.h:109-110); intersect1 still merges the kinds."""
    _, spec, R = case
    ref = RefScene(spec)
    ora = Oracle(spec)
    a = ora.intersect(R.origins, R.directions, R.tmin, R.tmax, any_hit=True)
    b = ref.intersect(R.origins, R.directions, R.tmin, R.tmax, any_hit=True)
    assert mismatches(a, b) == []
    # any-hit finds the same hit/miss set as closest-hit (only which hit is reported differs)
    c = ora.intersect(R.origins, R.directions, R.tmin, R.tmax)
    assert np.array_equal(a["hit"], c["hit"])


@needs_ref
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_product_builder_matches_reference(case):
    _, spec, _ = case
    ref = RefScene(spec)
    emu = EmuScene(spec)
    assert emu.geom_ids == ref.geom_ids
    for kind in spec.order:
        assert same_tree(emu.tree(kind), ref.tree(kind)) is None, kind


@needs_ref
def test_parallel_builder_matches_reference_on_large_mesh():
    """A 293,046-triangle grid: the product builder builds subtrees of 32,768 primitives or
    more on other threads and splices them back; the tree must still be the reference's node
    for node (DFS numbering, leaf order, boxes)."""
    wl = W.heightfield(n_rays=16, grid=384)
    ref = RefScene(wl.scene)
    emu = EmuScene(wl.scene)
    assert same_tree(emu.tree("mesh"), ref.tree("mesh")) is None


@needs_ref
@pytest.mark.parametrize("opts", [dict(min_leaf=1, max_depth=28, bins=64),
                                  dict(min_leaf=8, max_depth=6, bins=16),
                                  dict(min_leaf=2, max_depth=40, bins=3),
                                  dict(min_leaf=4, max_depth=28, bins=256)])
def test_build_options_match_reference(opts):
    wl = W.mixed_primitives(n_rays=10_000, n_spheres=2000, n_cylinders=200, n_planes=40, seed=4)
    ref, ora, emu = RefScene(wl.scene, **opts), Oracle(wl.scene, **opts), EmuScene(wl.scene, **opts)
    for kind in wl.scene.order:
        t = ref.tree(kind)
        assert same_tree(ora.tree(kind), t) is None
        assert same_tree(emu.tree(kind), t) is None
    R = wl.rays
    assert mismatches(ora.intersect(R.origins, R.directions),
                      ref.intersect(R.origins, R.directions)) == []


def test_reference_stack_depth_note():
    """Trees of the default options stay shallow enough that the reference's 28-entry stack
    (blazert/defines.h:6, blazert/datatypes.h:61-69) never overflows on these workloads: the
    stack peak the oracle records stays below 28."""
    wl = W.mixed_primitives(n_rays=50_000)
    out = Oracle(wl.scene).intersect(wl.rays.origins, wl.rays.directions, counters=True)
    assert out["stack_peak"].max() < 28


def test_build_statistics_match_the_reference():
    """The host builder's BVHBuildStatistics (tree_statistics over the tree bzr_commit keeps) equal
    the reference's own SAHBinnedBuilder::build statistics on every workload scene and edge
    case, with the default and two other option sets: depth, leaf and branch counts, primitives
    per leaf, and bad splits (one per failed partition attempt)."""
    from blazert_b200 import workloads as W
    from oracle.oracle import RefScene
    from tests.emu.emu import EmuScene
    from tests.scenes import edge_case_scenes

    specs = [W.mixed_primitives(n_rays=16, n_spheres=3000, n_cylinders=300, n_planes=30).scene,
             W.icosphere_pinhole().scene, W.adjoint_scene(n_rays=16).scene,
             W.batched_icospheres(n_scenes=2, seed=4, scale=0.01)[1].scene]
    specs += [spec for _, spec, _ in edge_case_scenes()]
    saw_bad = False
    for spec in specs:
        for kw in (dict(), dict(min_leaf=1, max_depth=40, bins=3), dict(min_leaf=8, max_depth=6, bins=16)):
            ref, emu = RefScene(spec, **kw), EmuScene(spec, **kw)
            for kind in spec.order:
                want, got = ref.build_statistics(kind), emu.build_statistics(kind)
                assert got == want, (kind, kw, got, want)
                saw_bad = saw_bad or want["bad_splits"] > 0
    assert saw_bad  # the icosphere meshes exercise the bad-split fallback
