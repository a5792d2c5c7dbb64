"""The GPU builder (bzr_commit_ex with BZR_COMMIT_GPU_BUILD) against the reference's own tree
and the host builder: the same nodes in the same DFS order (leaf flags, split axes, children,
leaf primitive lists bit for bit; boxes equal as values -- only the sign of a zero bound may
differ), and the same query results."""
import numpy as np
import pytest

from blazert_b200 import BuildOptions
from blazert_b200 import workloads as W
from oracle.oracle import Oracle, RefScene
from tests.helpers import mismatches, product_scene
from tests.scenes import edge_case_scenes

pytestmark = pytest.mark.gpu


def same_tree_values(a, b):
    """None when the trees match: integer arrays bit for bit, boxes by value."""
    for key in ("leaf", "axis", "children", "prim_cnt", "prim_ids", "bmin", "bmax"):
        x, y = a[key], b[key]
        if x.shape != y.shape:
            return f"{key}: shape {x.shape} vs {y.shape}"
        if not np.array_equal(x, y):
            return f"{key}: {int(np.count_nonzero(x != y))} entries differ"
    return None


def gpu_scene(spec, opts=None, gpu=True):
    import blazert_b200 as B

    s = B.Scene()
    for kind in spec.order:
        getattr(s, "add_" + kind)(*getattr(spec, kind).values())
    s.commit(opts, gpu_build=gpu)
    return s


def _cases():
    # the icosphere meshes have nodes whose cut sends everything to one side (bad splits:
    # next axis, or the middle of the range), the grid has none
    out = [("icosphere_pinhole", W.icosphere_pinhole()),
           ("mixed_primitives", W.mixed_primitives(n_rays=50_000)),
           ("heightfield_384", W.heightfield(n_rays=50_000, grid=384)),
           ("adjoint_scene", W.adjoint_scene(n_rays=50_000)),
           ("icosphere_level7", W.batched_icospheres(n_scenes=1, seed=4, scale=0.02)[0])]
    return out


@pytest.mark.parametrize("name,wl", _cases(), ids=lambda c: c if isinstance(c, str) else "")
def test_gpu_tree_is_the_reference_tree(name, wl):
    ref = RefScene(wl.scene)
    g = gpu_scene(wl.scene)
    h = gpu_scene(wl.scene, gpu=False)
    for kind in wl.scene.order:
        t = ref.tree(kind)
        t = dict(t, prim_cnt=t["prim_cnt"])
        assert same_tree_values(g.tree(kind), t) is None, kind
        assert same_tree_values(g.tree(kind), h.tree(kind)) is None, kind
        assert g.stats(kind)["max_depth"] == h.stats(kind)["max_depth"]
    R = wl.rays
    out = g.intersectN(R.origins, R.directions, R.tmin, R.tmax)
    assert mismatches(out, Oracle(wl.scene).intersect(R.origins, R.directions, R.tmin,
                                                      R.tmax)) == []


@pytest.mark.parametrize("opts", [dict(min_leaf=1, max_depth=28, bins=64),
                                  dict(min_leaf=8, max_depth=6, bins=16),
                                  dict(min_leaf=2, max_depth=40, bins=3),
                                  dict(min_leaf=4, max_depth=28, bins=256)])
def test_gpu_tree_build_options(opts):
    wl = W.mixed_primitives(n_rays=10_000, n_spheres=2000, n_cylinders=200, n_planes=40, seed=4)
    ref = RefScene(wl.scene, **opts)
    g = gpu_scene(wl.scene, BuildOptions(opts["min_leaf"], opts["max_depth"], opts["bins"]))
    for kind in wl.scene.order:
        assert same_tree_values(g.tree(kind), ref.tree(kind)) is None, (kind, opts)


@pytest.mark.parametrize("case", edge_case_scenes(), ids=lambda c: c[0])
def test_gpu_tree_edge_cases(case):
    """Edge-case scenes (degenerate, coincident, one primitive, huge coordinates...): the GPU
    builder gives the reference's tree, or, for non-finite inputs, the host builds it."""
    _, spec, R = case
    ref = RefScene(spec)
    g = gpu_scene(spec)
    for kind in spec.order:
        t = ref.tree(kind)
        if t is None or len(t["leaf"]) == 0:
            continue
        assert same_tree_values(g.tree(kind), t) is None, kind
    out = g.intersectN(R.origins, R.directions, R.tmin, R.tmax)
    assert mismatches(out, Oracle(spec).intersect(R.origins, R.directions, R.tmin, R.tmax)) == []


def test_gpu_build_on_a_large_mesh():
    """The 2,093,058-triangle grid: the device build (forced, and by default at this size)
    gives the host's tree and reports its time in the scene stats."""
    wl = W.heightfield(n_rays=16, grid=1024)
    gpu_scene(wl.scene)  # the first large build of a process also maps its device memory
    g = gpu_scene(wl.scene)
    h = gpu_scene(wl.scene, gpu=False)
    d = product_scene(wl.scene)  # the default builds this size on the device
    assert same_tree_values(g.tree("mesh"), h.tree("mesh")) is None
    assert same_tree_values(d.tree("mesh"), h.tree("mesh")) is None
    tg, th = g.stats("mesh")["build_seconds"], h.stats("mesh")["build_seconds"]
    print(f"build seconds: gpu {tg:.3f} host {th:.3f}")
    # the device build ran and was kept (a rejected device tree would add the host's time)
    assert tg < th


def test_build_statistics_through_the_c_abi():
    """bzr_scene_build_statistics of the device-built and host-built trees equal the reference's
    own BVHBuildStatistics (bad splits included: icosphere meshes)."""
    for wl in (W.icosphere_pinhole(), W.batched_icospheres(n_scenes=1, seed=4, scale=0.02)[0],
               W.mixed_primitives(n_rays=16)):
        ref = RefScene(wl.scene)
        for gpu in (True, False):
            s = gpu_scene(wl.scene, gpu=gpu)
            for kind in wl.scene.order:
                got = s.build_statistics(kind)
                want = ref.build_statistics(kind)
                assert {k: got[k] for k in want} == want, (kind, gpu)
                assert got["build_seconds"] >= 0.0
