"""The seeded synthetic workloads: sizes as specified, deterministic, well formed."""
import numpy as np

from blazert_b200 import workloads as W


def test_icosphere_counts_follow_the_reference_helper():
    # 20 * 4^k triangles; vertices are not de-duplicated (OriginSphere.h:56-64)
    for k, (nv, nf) in {0: (12, 20), 1: (72, 80), 4: (5112, 5120)}.items():
        v, f = W.icosphere(k)
        assert v.shape == (nv, 3) and f.shape == (nf, 3)
        assert f.max() < nv
        assert np.allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-15)


def test_pinhole_rays():
    wl = W.icosphere_pinhole()
    assert wl.rays.n == 512 * 512
    assert np.allclose(wl.rays.origins, [0, 0, 3])
    assert np.allclose(np.linalg.norm(wl.rays.directions, axis=1), 1.0)
    assert wl.meta["triangles"] == 5120


def test_mixed_primitives_deterministic():
    a, b = W.mixed_primitives(n_rays=1000), W.mixed_primitives(n_rays=1000)
    assert a.scene.order == ["spheres", "cylinders", "planes"]
    assert a.scene.spheres["centers"].shape == (10_000, 3)
    assert a.scene.cylinders["centers"].shape == (1_000, 3)
    assert a.scene.planes["centers"].shape == (100, 3)
    assert np.array_equal(a.rays.origins, b.rays.origins)
    assert np.array_equal(a.scene.cylinders["rotations"], b.scene.cylinders["rotations"])
    # rotations map e_z to the requested axis and are orthonormal
    R = a.scene.cylinders["rotations"]
    assert np.allclose(np.einsum("nij,nkj->nik", R, R), np.eye(3), atol=1e-12)
    r = a.scene.spheres["radii"]
    assert r.min() >= 0.1 and r.max() <= 2.0
