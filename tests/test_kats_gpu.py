"""The reference's known-answer vectors, the config samples and the golden render through the
CUDA path (C-ABI, host and device arrays): bit for bit equal to the reference's outputs."""
import numpy as np
import pytest

from blazert_b200 import workloads as W
from tests.helpers import (GOLDEN, golden_image_classes, image_classes, kat_spec, load_kats,
                           mismatches, product_scene, same_result, scene_primitives_workload)

pytestmark = pytest.mark.gpu

RECS = [r for r in load_kats()["records"] if r["check"] in ("intersect_primitive", "traverse", "scene")]


def test_kat_rays_through_cuda():
    bad = []
    for rec in RECS:
        want = rec["scene_result"] if rec["check"] != "scene" else rec["reference"]
        s = product_scene(kat_spec(rec))
        got = s.intersectN(np.array([rec["origin"]], float), np.array([rec["direction"]], float),
                           np.array([rec["tmin"]], float), np.array([rec["tmax"]], float))
        if not same_result(got, want):
            bad.append(rec["case"])
        s.close()
    assert bad == []


@pytest.mark.parametrize("name", ["icosphere_pinhole", "mixed_primitives"])
@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_config_samples_through_cuda(name, mode):
    g = np.load(f"{GOLDEN}/configs.npz")
    wl = W.WORKLOADS[name]()
    idx = g[f"{name}_idx"]
    R = wl.rays
    want = {k: g[f"{name}_{k}"] for k in ("t", "uv", "normal", "prim", "geom", "hit")}
    s = product_scene(wl.scene)
    got = s.intersectN(R.origins[idx], R.directions[idx], R.tmin[idx], R.tmax[idx], mode=mode)
    assert mismatches(got, want) == []


def test_golden_image_through_cuda():
    spec, R, (w, h) = scene_primitives_workload()
    s = product_scene(spec)
    got = s.intersectN(R.origins, R.directions)
    assert np.array_equal(image_classes(got, w, h), golden_image_classes())
