"""Shared helpers of the test suite."""
from __future__ import annotations

import numpy as np


def product_scene(spec, build_options=None):
    """blazert_b200.Scene built from a workloads.SceneSpec (kinds in the spec's add order)."""
    import blazert_b200 as B

    s = B.Scene()
    for kind in spec.order:
        getattr(s, "add_" + kind)(*getattr(spec, kind).values())
    s.commit(build_options)
    return s


def to_numpy(out):
    res = {}
    for k, v in out.items():
        if k.startswith("_"):
            continue
        res[k] = v.cpu().numpy() if hasattr(v, "cpu") else np.asarray(v)
    return res


def mismatches(got, ref):
    """Names of the result arrays that are not bit-identical to the reference's."""
    got = to_numpy(got)
    bad = []
    for k in ("hit", "prim", "geom"):
        a = got[k].view(np.uint8 if k == "hit" else np.uint32)
        if not np.array_equal(a, ref[k]):
            bad.append(f"{k}: {int(np.count_nonzero(a != ref[k]))} rays")
    for k in ("t", "uv", "normal"):
        a = np.ascontiguousarray(got[k]).view(np.uint64)
        b = np.ascontiguousarray(ref[k]).view(np.uint64)
        if not np.array_equal(a, b):
            bad.append(f"{k}: {int(np.count_nonzero((a != b).reshape(len(a), -1).any(1)))} rays")
    return bad


# ----------------------------------------------------------------------------- golden fixtures
import json as _json
import os as _os

GOLDEN = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "golden")


def load_kats():
    with open(_os.path.join(GOLDEN, "kats.json")) as f:
        return _json.load(f)


def kat_spec(rec):
    """SceneSpec of a captured KAT record (one collection, or the stored scene)."""
    from blazert_b200 import workloads as W

    if rec["check"] == "scene":
        s = W.SceneSpec()
        for kind in rec["scene"]["order"]:
            getattr(s, "add_" + kind)(*[np.asarray(v) for v in rec["scene"][kind].values()])
        return s
    k = rec["kind"]
    s = W.SceneSpec()
    if k == "mesh":
        s.add_mesh(np.array(rec["vertices"], float).reshape(-1, 3),
                   np.array(rec["faces"], np.uint32).reshape(-1, 3))
    elif k == "spheres":
        s.add_spheres(np.array(rec["centers"], float), np.array(rec["radii"], float))
    elif k == "planes":
        s.add_planes(np.array(rec["centers"], float), np.array(rec["dxs"], float),
                     np.array(rec["dys"], float), np.array(rec["rotations"], float).reshape(-1, 3, 3))
    else:
        # a few cylinder tests push a rotation more than they push cylinders; the collection
        # reads rotations[prim_id], so the first len(centers) entries are the ones in use
        n = len(rec["centers"])
        s.add_cylinders(np.array(rec["centers"], float), np.array(rec["semi_axes_a"], float)[:n],
                        np.array(rec["semi_axes_b"], float)[:n], np.array(rec["heights"], float)[:n],
                        np.array(rec["rotations"], float).reshape(-1, 3, 3)[:n])
    return s


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float64).view(np.uint64), np.asarray(b, np.float64).view(np.uint64))


def same_result(got, want, i=0):
    """got: batched outputs (numpy or torch); want: a fixture result dict."""
    got = to_numpy(got)
    return (bool(got["hit"][i]) == want["hit"]
            and int(got["prim"].view(np.uint32)[i]) == want["prim_id"]
            and int(got["geom"].view(np.uint32)[i]) == want.get("geom_id", int(got["geom"].view(np.uint32)[i]))
            and bits_equal(got["t"][i], want["distance"])
            and bits_equal(got["uv"][i], want["uv"])
            and bits_equal(got["normal"][i], want["normal"]))


def approx(x, v, eps=float(np.finfo(np.float32).eps) * 100, scale=1.0):
    """doctest::Approx, the tolerance of the reference's own tests."""
    return abs(x - v) < eps * (scale + max(abs(x), abs(v)))


def scene_primitives_workload():
    """examples/scene_primitives/main.cc:32-115: two cylinders (added first) and two spheres,
    1080 x 720 rays from (0, 5, 20) with directions (x/1080 - 0.5, y/720 - 0.5, -1)."""
    from blazert_b200 import workloads as W

    rot = np.array([[[0, 0, 1], [0, 1, 0], [-1, 0, 0]]], float).repeat(2, 0)
    s = W.SceneSpec()
    s.add_cylinders(np.array([[-3, 3, 0], [1, 4, 0]], float), np.array([1, 0.5]), np.array([1, 0.5]),
                    np.array([1, 2.0]), rot)
    s.add_spheres(np.array([[1, 1, 0], [-2, 10, 0]], float), np.array([0.5, 1.5]))
    w, h = 1080, 720
    y, x = np.meshgrid(np.arange(h, dtype=float), np.arange(w, dtype=float), indexing="ij")
    d = np.stack([x.ravel() / float(w) - 0.5, y.ravel() / float(h) - 0.5, -np.ones(w * h)], 1)
    o = np.broadcast_to([0.0, 5.0, 20.0], d.shape).copy()
    return s, W.RayBatch(o, d), (w, h)


def image_classes(out, w, h):
    """Pixel classes as the example writes them: row (h - y - 1); 1 red (prim 0), 2 green."""
    out = to_numpy(out)
    hit = out["hit"].reshape(h, w).astype(bool)
    prim0 = out["prim"].view(np.uint32).reshape(h, w) == 0
    cls = np.where(hit, np.where(prim0, 1, 2), 0)
    return cls[::-1]


def golden_image_classes():
    g = np.load(_os.path.join(GOLDEN, "scene_primitives_classes.npz"))
    hh, ww = g["shape"]
    n = hh * ww
    red = np.unpackbits(g["red"])[:n].reshape(hh, ww).astype(bool)
    green = np.unpackbits(g["green"])[:n].reshape(hh, ww).astype(bool)
    return np.where(red, 1, np.where(green, 2, 0))


def uncovered_workload(n_rays=200_000, seed=41):
    """All four kinds overlapping in space, with rays that the FP32 walk of the mixed mode does
    not cover mixed among ordinary ones (a mixed pass hands them to its FP64 pass): axis
    directions (two zero components), one zero component, a component of 1e-13 (its inverse is
    above 2^40), an origin 2e18 back along the ray, and ordinary rays.  Returns the workload and
    the class of each ray (0 ordinary, 1 axis, 2 one zero, 3 tiny, 4 far origin)."""
    from blazert_b200 import workloads as W

    wl = W.mixed_primitives(n_rays=n_rays, n_spheres=2000, n_cylinders=400, n_planes=60, seed=seed)
    v, f = W.icosphere(3)
    spec = W.SceneSpec().add_mesh(v * 60.0, f)
    for k in wl.scene.order:
        getattr(spec, "add_" + k)(*getattr(wl.scene, k).values())
    rng = np.random.default_rng(seed)
    o, d = wl.rays.origins.copy(), wl.rays.directions.copy()
    cls = rng.integers(0, 5, n_rays)
    rows = np.arange(n_rays)
    big, small = np.argmax(np.abs(d), 1), np.argmin(np.abs(d), 1)
    axis = np.zeros_like(d)
    axis[rows, big] = np.sign(d[rows, big])
    d = np.where((cls == 1)[:, None], axis, d)
    one = cls == 2
    d[rows[one], small[one]] = 0.0
    tiny = cls == 3
    d[rows[tiny], small[tiny]] = np.copysign(1e-13, d[rows[tiny], small[tiny]])
    far = cls == 4
    o[far] = o[far] - 2e18 * d[far]
    rays = W.RayBatch(o, d, np.zeros(n_rays), np.full(n_rays, np.inf))
    return W.Workload("uncovered_rays", spec, rays, {}), cls
