"""The reference's own known-answer vectors (tests/golden/kats.json, captured from the
reference's test files by oracle/_ref/kat_runner) against the CPU oracle, the product's host
precompute and the kernels' code run by the CPU emulator.  Results must equal the reference's
outputs bit for bit; the reference's outputs themselves satisfy the tests' Approx checks."""
import numpy as np
import pytest

from blazert_b200 import workloads as W
from oracle.oracle import Oracle
from tests.emu.emu import EmuScene, box_accept
from tests.helpers import (approx, bits_equal, golden_image_classes, image_classes, kat_spec,
                           load_kats, same_result, scene_primitives_workload, mismatches, GOLDEN)

KATS = load_kats()
RECS = KATS["records"]
RAY_RECS = [r for r in RECS if r["check"] in ("intersect_primitive", "traverse", "scene")]


def test_capture_is_complete():
    s = KATS["summary"]
    assert s["failed"] == 0 and s["checks"] > 4000
    kinds = {(r["check"], r.get("kind")) for r in RECS}
    for k in ("mesh", "spheres", "planes", "cylinders"):
        assert ("intersect_primitive", k) in kinds and ("traverse", k) in kinds
    assert sum(r["check"] == "intersect_node" for r in RECS) == 8
    assert sum(r["check"] == "scene" for r in RECS) == 4


def test_reference_outputs_meet_the_tests_expectations():
    """Sanity of the capture: the stored reference outputs pass the assertions they came from."""
    for r in RECS:
        if r["check"] == "intersect_primitive" or (r["check"] == "traverse" and r["expected"]["mode"] < 3):
            e, got = r["expected"], r["reference"]
            assert got["hit"] == e["hit"], r["case"]
            assert approx(got["distance"], e["distance"]), r["case"]
        if r["check"] == "scene":
            e, got = r["expected"], r["reference"]
            assert got["hit"] == e["hit"] and got["geom_id"] == e["geom_id"]
            assert approx(got["distance"], e["distance"])
            assert all(approx(a, b) for a, b in zip(got["normal"], e["normal"]))


@pytest.mark.parametrize("rec", [r for r in RECS if r["check"] == "intersect_primitive"],
                         ids=lambda r: r["case"][-60:])
def test_oracle_primitive_tests(rec):
    ora = Oracle(kat_spec(rec))
    got = ora.primitive0(rec["kind"], rec["origin"], rec["direction"], rec["tmin"], rec["tmax"])
    want = rec["reference"]
    assert got["hit"] == want["hit"] and got["prim"] == want["prim_id"]
    assert bits_equal(got["t"], want["distance"]) and bits_equal(got["normal"], want["normal"])
    assert bits_equal(got["uv"], want["uv"])


@pytest.mark.parametrize("rec", [r for r in RECS if r["check"] == "traverse"],
                         ids=lambda r: r["case"][-60:])
def test_oracle_traversals(rec):
    ora = Oracle(kat_spec(rec))
    got = ora.traverse(rec["kind"], rec["origin"], rec["direction"], rec["tmin"], rec["tmax"])
    want = rec["reference"]
    assert got["hit"] == want["hit"] and got["prim"] == want["prim_id"]
    assert bits_equal(got["t"], want["distance"]) and bits_equal(got["normal"], want["normal"])


def _batch(rec):
    return (np.array([rec["origin"]], float), np.array([rec["direction"]], float),
            np.array([rec["tmin"]], float), np.array([rec["tmax"]], float))


def test_scene_results_oracle_and_emulator():
    """intersect1 on a scene holding only the test's collection: the oracle and the kernels'
    code must return the reference's result bit for bit."""
    for rec in RAY_RECS:
        want = rec["scene_result"] if rec["check"] != "scene" else rec["reference"]
        spec = kat_spec(rec)
        for impl in (Oracle(spec), EmuScene(spec)):
            got = impl.intersect(*_batch(rec))
            assert same_result(got, want), (type(impl).__name__, rec["case"])


def test_node_slab_tests():
    for rec in [r for r in RECS if r["check"] == "intersect_node"]:
        want = rec["reference"]
        h, tmin, tmax = Oracle.intersect_node(rec["in"][0], rec["in"][1], rec["bmin"], rec["bmax"],
                                              rec["origin"], rec["direction"])
        assert h == want["hit"] and bits_equal(tmin, want["tmin"]) and bits_equal(tmax, want["tmax"]), rec["case"]
        assert box_accept(rec["bmin"], rec["bmax"], rec["origin"], rec["direction"],
                          rec["in"][0], rec["in"][1]) == want["hit"], rec["case"]


def test_boxes_and_centres_of_the_product_precompute():
    for rec in [r for r in RECS if r["check"] in ("bounding_box", "center")]:
        mn, mx, c = EmuScene(kat_spec(rec)).prim_box(rec["kind"], rec["prim_id"])
        if rec["check"] == "bounding_box":
            assert bits_equal(mn, rec["reference"]["min"]) and bits_equal(mx, rec["reference"]["max"])
        else:
            assert bits_equal(c, rec["reference"])


@pytest.mark.parametrize("name", ["icosphere_pinhole", "mixed_primitives"])
def test_config_samples(name):
    import hashlib

    g = np.load(f"{GOLDEN}/configs.npz")
    wl = W.WORKLOADS[name]()
    R = wl.rays
    h = hashlib.sha256()
    arrays = ((wl.scene.mesh["vertices"], wl.scene.mesh["faces"]) if name == "icosphere_pinhole" else
              (wl.scene.spheres["centers"], wl.scene.cylinders["rotations"], wl.scene.planes["rotations"]))
    for a in arrays + (R.origins, R.directions):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.digest() == g[f"{name}_digest"].tobytes(), "workload generator changed"
    idx = g[f"{name}_idx"]
    want = {k: g[f"{name}_{k}"] for k in ("t", "uv", "normal", "prim", "geom", "hit")}
    got = Oracle(wl.scene).intersect(R.origins[idx], R.directions[idx], R.tmin[idx], R.tmax[idx])
    assert mismatches(got, want) == []


def test_golden_image_classes():
    spec, R, (w, h) = scene_primitives_workload()
    got = Oracle(spec).intersect(R.origins, R.directions)
    assert np.array_equal(image_classes(got, w, h), golden_image_classes())
