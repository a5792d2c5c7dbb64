"""Distance to surface and the nearest-surface query on the CPU.

* the oracle's C restatement (oracle/bzr_oracle.c) against the reference's own
  distance_to_surface and closest_point_on_triangle (oracle/_ref) on seeded points;
* the reference test suite's known-answer distances (tests/golden/kats.json, 255 asserts of
  test_sphere.cpp, test_plane.cpp, test_cylinder.cpp) against the oracle and the kernels' code;
* the kernels' per-point code (blazert_b200/csrc/distance_core.cuh compiled for the CPU by
  tests/emu) against both, including the BVH-pruned nearest-surface search against an
  exhaustive loop: ties, NaN distances and trees deeper than the search stack."""
import numpy as np
import pytest

from blazert_b200 import workloads as W
from oracle.oracle import Oracle, RefScene
from tests.emu.emu import EmuScene
from tests.helpers import approx, bits_equal, kat_spec, load_kats
from tests.scenes import distance_queries, edge_case_scenes

DIST_RECS = [r for r in load_kats()["records"] if r["check"] == "distance_to_surface"]


def test_capture_holds_the_distance_asserts():
    kinds = {r["kind"] for r in DIST_RECS}
    assert kinds == {"spheres", "planes", "cylinders"}
    assert len(DIST_RECS) == 255
    for r in DIST_RECS:  # the reference's outputs pass the test's own Approx check
        assert approx(r["reference"], r["expected"]), r["case"]


@pytest.mark.parametrize("impl", ["oracle", "emu"])
def test_known_answer_distances(impl):
    bad = []
    for r in DIST_RECS:
        spec = kat_spec(r)
        s = Oracle(spec) if impl == "oracle" else EmuScene(spec)
        d, _ = s.distance_to_surface(r["kind"], [r["prim_id"]], np.array([r["point"]], float))
        if not bits_equal(d[0], r["reference"]):
            bad.append((r["case"], r["point"], float(d[0]), r["reference"]))
    assert bad == []


def _scenes():
    return [("mixed", W.mixed_primitives(n_rays=16, n_spheres=600, n_cylinders=400, n_planes=60,
                                         seed=7).scene),
            ("icosphere", W.icosphere_pinhole().scene),
            ("adjoint", W.adjoint_scene(n_rays=16).scene)] + \
        [(name, spec) for name, spec, _ in edge_case_scenes()]


@pytest.mark.parametrize("name,spec", _scenes(), ids=lambda x: x if isinstance(x, str) else "")
def test_per_primitive_distances_pinned(name, spec):
    """oracle == reference == the kernels' code, bit for bit, per kind."""
    rng = np.random.default_rng(5)
    ora, ref, emu = Oracle(spec), RefScene(spec), EmuScene(spec)
    for kind in spec.order:
        ids, pts = distance_queries(spec, kind, rng, 4000)
        a, ac = ora.distance_to_surface(kind, ids, pts)
        b, bc = ref.distance_to_surface(kind, ids, pts)
        c, cc = emu.distance_to_surface(kind, ids, pts)
        assert bits_equal(a, b), (name, kind)
        assert bits_equal(c, b), (name, kind)
        if kind == "mesh":
            assert bits_equal(ac, bc) and bits_equal(cc, bc), name


@pytest.mark.parametrize("name,spec", _scenes(), ids=lambda x: x if isinstance(x, str) else "")
def test_nearest_surface_equals_exhaustion(name, spec):
    rng = np.random.default_rng(9)
    lo = min(np.min(getattr(spec, k)["centers" if k != "mesh" else "vertices"]) for k in spec.order)
    hi = max(np.max(getattr(spec, k)["centers" if k != "mesh" else "vertices"]) for k in spec.order)
    span = hi - lo
    pts = rng.uniform(lo - 0.2 * span, hi + 0.2 * span, (1500, 3))
    # and points right at primitives (ties between neighbours, zero distances)
    for kind in spec.order:
        pts = np.concatenate([pts, distance_queries(spec, kind, rng, 300)[1]])
    want = Oracle(spec).closest_surface(pts)
    got = EmuScene(spec).closest_surface(pts)
    assert bits_equal(got["distance"], want["distance"]), name
    assert np.array_equal(got["prim"], want["prim"]) and np.array_equal(got["geom"], want["geom"])


def test_nearest_surface_ties_and_kind_order():
    """Equal distances: the lowest id within a kind, the first kind across kinds; degenerate
    triangles (NaN distances) never win."""
    c = np.array([[0.0, 0, 0], [5.0, 0, 0], [0.0, 0, 0], [5.0, 0, 0]])  # ids 2, 3 duplicate 0, 1
    r = np.array([1.0, 1.0, 1.0, 1.0])
    v = np.array([[2.5, -1, -1], [2.5, 1, -1], [2.5, 0, 1], [2.5, 0, 0], [2.5, 0, 0], [2.5, 0, 0]])
    f = np.array([[3, 4, 5], [0, 1, 2]], np.uint32)  # face 0 degenerate (one point)
    spec = W.SceneSpec().add_spheres(c, r).add_mesh(v, f)  # spheres geom 0, mesh geom 1
    pts = np.array([[0.0, 0, 3], [5.0, 0, 3], [1.75, 0, 0], [2.5, 0, 5], [-3.0, 0, 0]])
    want = Oracle(spec).closest_surface(pts)
    got = EmuScene(spec).closest_surface(pts)
    assert bits_equal(got["distance"], want["distance"])
    assert np.array_equal(got["prim"], want["prim"]) and np.array_equal(got["geom"], want["geom"])
    # (1.75, 0, 0): 0.75 to sphere 0 and to the triangle plane x = 2.5 -- the mesh comes first
    assert want["distance"][2] == 0.75 and want["geom"][2] == 1 and want["prim"][2] == 1
    assert want["prim"][0] == 0 and want["prim"][1] == 1  # lowest of the duplicate ids


def test_nearest_surface_on_a_tree_deeper_than_the_search_stack():
    """Spheres at exponentially growing positions with 2 bins make a tree 70 levels deep (with
    max_tree_depth raised): the search evaluates that kind exhaustively and still matches."""
    n = 90
    c = np.stack([2.0 ** np.arange(n), np.zeros(n), np.zeros(n)], 1)
    spec = W.SceneSpec().add_spheres(c, np.full(n, 0.25))
    kw = dict(min_leaf=1, max_depth=200, bins=2)
    emu = EmuScene(spec, **kw)
    t = emu.tree("spheres")
    depth = np.zeros(len(t["leaf"]), int)
    for i in range(len(t["leaf"])):
        if t["leaf"][i] != 1:
            depth[t["children"][i]] = depth[i] + 1
    assert depth.max() > 64
    pts = np.concatenate([c[::7] + [0.0, 1.0, 0.0], [[3.0, 0.0, 0.0], [1e20, 5.0, 0.0]]])
    want = Oracle(spec, **kw).closest_surface(pts)
    got = emu.closest_surface(pts)
    assert bits_equal(got["distance"], want["distance"])
    assert np.array_equal(got["prim"], want["prim"])


def test_bad_primitive_id_gives_nan_and_the_error_bit():
    spec = W.SceneSpec().add_spheres(np.zeros((2, 3)), np.ones(2))
    emu = EmuScene(spec)
    import ctypes as C
    from oracle.oracle import _dp, _ptr, _u32p
    ids = np.array([0, 7], np.uint32)
    pts = np.zeros((2, 3))
    out = np.empty(2)
    err = emu._lib.emu_distance_to_surface(emu._h, 1, 2, _ptr(ids, _u32p), _ptr(pts, _dp),
                                           _ptr(out, _dp), None)
    assert out[0] == 1.0 and np.isnan(out[1]) and err == 4


def same_or_both_nan(a, b):
    """Bit-identical, or NaN on both sides (the default NaN's sign differs between x86 and the
    GPU)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    nan = np.isnan(a) & np.isnan(b)
    return bool(np.array_equal(np.isnan(a), np.isnan(b))) and bits_equal(a[~nan], b[~nan])


def degenerate_scene():
    """Primitives at the edges of the reference's formulas: zero semi-axes and heights,
    flat and huge cylinders, zero-size and rotated planes, collinear and repeated-vertex
    triangles, a zero-radius sphere, coordinates of 1e150."""
    rot = W.rotation_to(np.array([[0, 0, 1.0], [1.0, 0, 0], [0, 1.0, 1.0], [1, 2, 3.0],
                                  [0, 0, 1.0], [0, 0, 1.0]]))
    cyl = dict(c=np.array([[0, 0, 0], [5, 0, 0], [0, 5, 0], [1e150, 0, 0], [0, 0, 5], [9, 9, 9.0]]),
               a=np.array([0.0, 1.0, 0.5, 2.0, 1.0, 0.0]), b=np.array([0.0, 1.0, 2.0, 2.0, 1e-300, 1.0]),
               h=np.array([2.0, 0.0, 1.0, 3.0, 1.0, 0.0]))
    v = np.array([[0, 0, 0], [1, 1, 1], [2, 2, 2], [0, 0, 0], [1, 0, 0], [0, 1, 0.0],
                  [1e150, 0, 0], [1e150, 1e150, 0], [0, 0, 1e150]])
    f = np.array([[0, 1, 2], [0, 0, 0], [3, 4, 5], [6, 7, 8], [3, 3, 4]], np.uint32)
    return (W.SceneSpec().add_mesh(v, f)
            .add_spheres(np.array([[0, 0, 0], [1e150, 1e150, 1e150], [3, 3, 3.0]]), np.array([0.0, 1.0, 1e-200]))
            .add_planes(np.array([[0, 0, 0], [2, 2, 2], [1e150, 0, 0.0]]), np.array([0.0, 1.0, 1e150]),
                        np.array([0.0, 2.0, 3.0]), W.rotation_to(np.array([[0, 0, 1.0], [1, 1, 1.0], [0, 1.0, 0]])))
            .add_cylinders(cyl["c"], cyl["a"], cyl["b"], cyl["h"], rot))


def _degenerate_points(spec, kind, rng):
    col = getattr(spec, kind)
    n = len(col["faces"]) if kind == "mesh" else len(col["centers"])
    special = np.array([[0, 0, 0], [0, 0, 1], [0, 0, -1], [1, 0, 0], [0, 1, 0], [0.5, 0.5, 0.5],
                        [1e150, 0, 0], [-1e150, 1e150, 0], [5, 0, 0], [5, 0, 1e-300], [9, 9, 9.0],
                        [np.inf, 0, 0], [0, np.nan, 0], [0, 0, 5.5]])
    ids = np.repeat(np.arange(n, dtype=np.uint32), len(special))
    pts = np.tile(special, (n, 1))
    more_ids, more_pts = distance_queries(spec, kind, rng, 400)
    return np.concatenate([ids, more_ids]), np.concatenate([pts, more_pts])


def test_degenerate_primitives_and_points():
    spec = degenerate_scene()
    rng = np.random.default_rng(17)
    ora, ref, emu = Oracle(spec), RefScene(spec), EmuScene(spec)
    for kind in spec.order:
        ids, pts = _degenerate_points(spec, kind, rng)
        a, ac = ora.distance_to_surface(kind, ids, pts)
        b, bc = ref.distance_to_surface(kind, ids, pts)
        c, cc = emu.distance_to_surface(kind, ids, pts)
        assert same_or_both_nan(a, b), kind
        assert same_or_both_nan(c, b), kind
        if kind == "mesh":
            assert same_or_both_nan(ac, bc) and same_or_both_nan(cc, bc)
    pts = np.concatenate([_degenerate_points(spec, k, rng)[1] for k in spec.order])
    want, got = Oracle(spec).closest_surface(pts), emu.closest_surface(pts)
    assert same_or_both_nan(got["distance"], want["distance"])
    assert np.array_equal(got["prim"], want["prim"]) and np.array_equal(got["geom"], want["geom"])
