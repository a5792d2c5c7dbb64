"""Distance queries through the product (bzr_distance_to_surface, bzr_closest_surface) on the
GPU against the oracle and the reference's own outputs, bit for bit: the reference test suite's
known-answer distances, seeded points on every kind of several scenes (host and device arrays),
the BVH-pruned nearest-surface search against exhaustion, and the error behaviour."""
import numpy as np
import pytest

import blazert_b200 as B
from blazert_b200 import workloads as W
from oracle.oracle import Oracle
from tests.helpers import bits_equal, kat_spec, load_kats, product_scene
from tests.scenes import distance_queries, edge_case_scenes

pytestmark = pytest.mark.gpu

DIST_RECS = [r for r in load_kats()["records"] if r["check"] == "distance_to_surface"]


def test_known_answer_distances_on_the_gpu():
    bad = []
    for r in DIST_RECS:
        s = product_scene(kat_spec(r))
        d = s.distance_to_surface(r["kind"], [r["prim_id"]], np.array([r["point"]], float))
        if not bits_equal(d[0], r["reference"]):
            bad.append((r["case"], float(d[0]), r["reference"]))
    assert bad == []


def _scenes():
    return [("mixed", W.mixed_primitives(n_rays=16, seed=2).scene),
            ("icosphere", W.icosphere_pinhole().scene),
            ("adjoint", W.adjoint_scene(n_rays=16).scene),
            ("heightfield_256", W.heightfield(n_rays=16, grid=256).scene)] + \
        [(name, spec) for name, spec, _ in edge_case_scenes()]


@pytest.mark.parametrize("name,spec", _scenes(), ids=lambda x: x if isinstance(x, str) else "")
def test_per_primitive_distances(name, spec):
    import torch

    rng = np.random.default_rng(21)
    s, ora = product_scene(spec), Oracle(spec)
    for kind in spec.order:
        ids, pts = distance_queries(spec, kind, rng, 20000)
        want, want_c = ora.distance_to_surface(kind, ids, pts)
        got = s.distance_to_surface(kind, ids, pts, closest=kind == "mesh")
        if kind == "mesh":
            got, got_c = got
            assert bits_equal(got_c, want_c), name
        assert bits_equal(got, want), (name, kind)
        dev = s.distance_to_surface(kind, torch.from_numpy(ids.astype(np.int32)).cuda(),
                                    torch.from_numpy(pts).cuda())
        torch.cuda.synchronize()
        assert bits_equal(dev.cpu().numpy(), want), (name, kind)
    assert s.check() == 0


@pytest.mark.parametrize("name,spec", _scenes(), ids=lambda x: x if isinstance(x, str) else "")
def test_closest_surface(name, spec):
    import torch

    rng = np.random.default_rng(22)
    arrays = [getattr(spec, k)["centers" if k != "mesh" else "vertices"] for k in spec.order]
    lo = min(float(a.min()) for a in arrays)
    hi = max(float(a.max()) for a in arrays)
    pts = rng.uniform(lo - 0.2 * (hi - lo), hi + 0.2 * (hi - lo), (3000, 3))
    for kind in spec.order:
        pts = np.concatenate([pts, distance_queries(spec, kind, rng, 500)[1]])
    want = Oracle(spec).closest_surface(pts)
    s = product_scene(spec)
    got = s.closest_surface(pts)
    assert bits_equal(got["distance"], want["distance"]), name
    assert np.array_equal(got["prim"], want["prim"]) and np.array_equal(got["geom"], want["geom"])
    dev = s.closest_surface(torch.from_numpy(pts).cuda())
    torch.cuda.synchronize()
    assert bits_equal(dev["distance"].cpu().numpy(), want["distance"])
    assert np.array_equal(dev["prim"].cpu().numpy().view(np.uint32), want["prim"])


def test_distance_errors():
    import torch

    spec = W.SceneSpec().add_spheres(np.zeros((3, 3)), np.ones(3))
    s = product_scene(spec)
    with pytest.raises(B.BlazertError) as e:  # host arrays: checked before the launch
        s.distance_to_surface("spheres", [0, 3], np.zeros((2, 3)))
    assert e.value.code == B.EINVAL
    with pytest.raises(B.BlazertError):  # a kind the scene does not hold
        s.distance_to_surface("planes", [0], np.zeros((1, 3)))
    with pytest.raises(ValueError):
        s.distance_to_surface("spheres", [0], np.zeros((1, 3)), closest=True)
    assert s.distance_to_surface("spheres", [], np.zeros((0, 3))).shape == (0,)
    # device arrays: NaN for the bad id, and the scene's error word records it
    d = s.distance_to_surface("spheres", torch.tensor([1, 9], dtype=torch.int32, device="cuda"),
                              torch.zeros((2, 3), dtype=torch.float64, device="cuda"))
    torch.cuda.synchronize()
    out = d.cpu().numpy()
    assert out[0] == 1.0 and np.isnan(out[1])
    with pytest.raises(B.BlazertError) as e:
        s.check()
    assert e.value.code == B.EDEVICE_FLAG


def test_closest_surface_large_batch_is_sorted_and_exact():
    """From 65,536 points on, the batch is processed in Morton order (a device counting sort);
    every point's result is still its own, equal to the CPU copy of the kernels' search."""
    from tests.emu.emu import EmuScene

    wl = W.closest_surface_points(n_points=70_000)
    pts = wl.meta["points"]
    s = product_scene(wl.scene)
    got = s.closest_surface(pts)
    want = EmuScene(wl.scene).closest_surface(pts)
    assert bits_equal(got["distance"], want["distance"])
    assert np.array_equal(got["prim"], want["prim"]) and np.array_equal(got["geom"], want["geom"])


def test_degenerate_primitives_and_points_on_the_gpu():
    """The degenerate scene and points of the CPU test through the product: bit for bit, NaN
    where the oracle gives NaN."""
    from tests.test_distance import _degenerate_points, degenerate_scene, same_or_both_nan

    spec = degenerate_scene()
    rng = np.random.default_rng(17)
    s, ora = product_scene(spec), Oracle(spec)
    all_pts = []
    for kind in spec.order:
        ids, pts = _degenerate_points(spec, kind, rng)
        all_pts.append(pts)
        want, want_c = ora.distance_to_surface(kind, ids, pts)
        got = s.distance_to_surface(kind, ids, pts, closest=kind == "mesh")
        if kind == "mesh":
            got, got_c = got
            assert same_or_both_nan(got_c, want_c)
        assert same_or_both_nan(got, want), kind
    pts = np.concatenate(all_pts)
    want = ora.closest_surface(pts)
    got = s.closest_surface(pts)
    assert same_or_both_nan(got["distance"], want["distance"])
    assert np.array_equal(got["prim"], want["prim"]) and np.array_equal(got["geom"], want["geom"])


def test_large_host_batches_are_pipelined_and_exact():
    """Host-array batches above 262,144 queries run as a pipeline of chunks (copies in, kernels
    and copies out overlapping): every chunk's results land at their own indices."""
    from tests.emu.emu import EmuScene

    wl = W.mixed_primitives(n_rays=16, seed=4)
    s, ora = product_scene(wl.scene), Oracle(wl.scene)
    rng = np.random.default_rng(31)
    for kind in ("spheres", "planes"):
        ids, pts = distance_queries(wl.scene, kind, rng, 700_000)
        assert bits_equal(s.distance_to_surface(kind, ids, pts),
                          ora.distance_to_surface(kind, ids, pts)[0]), kind
    near = W.closest_surface_points(n_points=600_000)
    s2 = product_scene(near.scene)
    got = s2.closest_surface(near.meta["points"])
    want = EmuScene(near.scene).closest_surface(near.meta["points"])
    assert bits_equal(got["distance"], want["distance"])
    assert np.array_equal(got["prim"], want["prim"]) and np.array_equal(got["geom"], want["geom"])
