"""The persistent scene format through the product (bzr_scene_save / bzr_scene_load,
bzr_scene_serialize / bzr_scene_deserialize) on the GPU: a loaded scene answers rays and
distance queries bit for bit as the saved one (and as the oracle), files written by the CPU
emulator's copy of the same code load in the product, the device-built tree of the 2M-triangle
grid survives the round trip, and damaged files are refused with BZR_EINVAL."""
import numpy as np
import pytest

import blazert_b200 as B
from blazert_b200 import workloads as W
from oracle.oracle import Oracle
from tests.emu.emu import EmuScene
from tests.helpers import bits_equal, mismatches, product_scene
from tests.scenes import distance_queries, edge_case_scenes

pytestmark = pytest.mark.gpu


def _cases():
    out = [("mixed", W.mixed_primitives(n_rays=100_000)), ("adjoint", W.adjoint_scene(n_rays=100_000)),
           ("icosphere", W.icosphere_pinhole())]
    out += [(name, W.Workload(name, spec, R, {})) for name, spec, R in edge_case_scenes()]
    return out


@pytest.mark.parametrize("name,wl", _cases(), ids=lambda x: x if isinstance(x, str) else "")
def test_saved_scene_answers_as_the_original(name, wl, tmp_path):
    spec, R = wl.scene, wl.rays
    a = product_scene(spec)
    path = tmp_path / f"{name}.bzrscene"
    a.save(path)
    b = B.Scene.load(path)
    ra = a.intersectN(R.origins, R.directions, R.tmin, R.tmax)
    rb = b.intersectN(R.origins, R.directions, R.tmin, R.tmax)
    for k in ("t", "uv", "normal", "prim", "geom", "hit"):
        assert np.array_equal(ra[k].view(np.uint8), rb[k].view(np.uint8)), k
    assert mismatches(rb, Oracle(spec).intersect(R.origins, R.directions, R.tmin, R.tmax)) == []
    rng = np.random.default_rng(4)
    for kind in spec.order:
        ids, pts = distance_queries(spec, kind, rng, 2000)
        assert bits_equal(a.distance_to_surface(kind, ids, pts), b.distance_to_surface(kind, ids, pts))
    assert b.to_bytes() == a.to_bytes()
    for kind in spec.order:
        assert b.stats(kind)["max_depth"] == a.stats(kind)["max_depth"]


def test_emulator_files_load_in_the_product():
    wl = W.mixed_primitives(n_rays=50_000, seed=9)
    data = EmuScene(wl.scene).encode()
    s = B.Scene.from_bytes(data)
    R = wl.rays
    assert mismatches(s.intersectN(R.origins, R.directions, R.tmin, R.tmax),
                      Oracle(wl.scene).intersect(R.origins, R.directions, R.tmin, R.tmax)) == []
    assert s.to_bytes() == data


def test_device_built_tree_round_trip(tmp_path):
    wl = W.heightfield(n_rays=200_000, grid=1024)
    a = product_scene(wl.scene)  # 2,093,058 triangles: built on the device
    a.save(tmp_path / "grid.bzrscene")
    b = B.Scene.load(tmp_path / "grid.bzrscene")
    R = wl.rays
    ra = a.intersectN(R.origins, R.directions, R.tmin, R.tmax)
    rb = b.intersectN(R.origins, R.directions, R.tmin, R.tmax)
    for k in ("t", "prim", "hit"):
        assert np.array_equal(ra[k].view(np.uint8), rb[k].view(np.uint8)), k


def test_damaged_files_are_refused(tmp_path):
    s = product_scene(W.mixed_primitives(n_rays=10, n_spheres=50, n_cylinders=5, n_planes=2).scene)
    data = bytearray(s.to_bytes())
    data[len(data) // 2] ^= 0x10
    p = tmp_path / "bad.bzrscene"
    p.write_bytes(bytes(data))
    with pytest.raises(B.BlazertError) as e:
        B.Scene.load(p)
    assert e.value.code == B.EINVAL and "checksum" in str(e.value)
    with pytest.raises(B.BlazertError):
        B.Scene.load(tmp_path / "missing.bzrscene")
    with pytest.raises(B.BlazertError) as e:
        B.Scene().to_bytes()  # not committed
    assert e.value.code == B.ESTATE
