#!/usr/bin/env python3
"""Regenerates the golden fixtures in tests/golden/ from the reference (run where the reference
sources are; the fixtures are committed so the tests do not need them).

    make -C oracle all && python tests/golden/make_golden.py [--reference DIR]

DIR defaults to the directory "reference" beside this repository.

kats.json
    Every known-answer vector the reference's own test files assert for the double-precision
    hot path, captured by oracle/_ref/kat_runner (the test files compiled unchanged against
    the doctest and blaze shims, oracle/kat/capture.h): primitive tests, traversals, node slab
    tests, boxes and centres -- each with the test's expected values and the reference's own
    outputs -- plus the four scene-level cases of test/test_scene.cpp:20-166 restated here.
    For every ray case it also stores "scene_result": intersect1 of the reference on a scene
    holding only that collection (what the GPU path must return bit for bit).
configs.npz
    Reference intersect1 outputs (oracle/_ref/libref_parity.so) on deterministic samples of the
    icosphere-pinhole and mixed-primitive workloads, with a digest of the input arrays.
scene_primitives_classes.npz
    The golden render examples/baseline/scene_primitives.png of the reference (produced by
    examples/scene_primitives/main.cc:32-115) reduced to its pixel classes: 0 miss (black),
    1 prim_id 0 (red), 2 other hit (green), bit-packed.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from blazert_b200 import workloads as W  # noqa: E402
from oracle.oracle import RefScene  # noqa: E402

DBL_MAX = float(np.finfo(np.float64).max)


def spec_of(rec):
    s = W.SceneSpec()
    k = rec["kind"]
    if k == "mesh":
        s.add_mesh(np.array(rec["vertices"], float).reshape(-1, 3), np.array(rec["faces"], np.uint32).reshape(-1, 3))
    elif k == "spheres":
        s.add_spheres(np.array(rec["centers"], float), np.array(rec["radii"], float))
    elif k == "planes":
        s.add_planes(np.array(rec["centers"], float), np.array(rec["dxs"], float),
                     np.array(rec["dys"], float), np.array(rec["rotations"], float).reshape(-1, 3, 3))
    else:
        s.add_cylinders(np.array(rec["centers"], float), np.array(rec["semi_axes_a"], float),
                        np.array(rec["semi_axes_b"], float), np.array(rec["heights"], float),
                        np.array(rec["rotations"], float).reshape(-1, 3, 3))
    return s


def result_dict(out, i=0):
    return {"hit": bool(out["hit"][i]), "prim_id": int(out["prim"][i]), "geom_id": int(out["geom"][i]),
            "distance": float(out["t"][i]), "uv": [float(x) for x in out["uv"][i]],
            "normal": [float(x) for x in out["normal"][i]]}


def scene_cases():
    """test/test_scene.cpp:20-166 (double instantiation), restated: scene, ray, expected."""
    I = np.eye(3)[None]
    cases = []
    s = W.SceneSpec().add_spheres(np.array([[0.0, 0, 0]]), np.array([1.0]))
    cases.append(("Scene with Sphere", s, [2, 0, 0], [-1, 0, 0],
                  dict(hit=True, geom_id=0, distance=1.0, normal=[1, 0, 0])))
    s = W.SceneSpec().add_planes(np.array([[0.0, 0, 0]]), np.array([2.0]), np.array([2.0]), I)
    cases.append(("Scene with Plane", s, [0, 0, 5], [0, 0, -1],
                  dict(hit=True, geom_id=0, distance=5.0, normal=[0, 0, 1])))
    s = W.SceneSpec().add_cylinders(np.array([[0.0, 0, 0]]), np.array([2.0]), np.array([2.0]),
                                    np.array([2.0]), I)
    cases.append(("Scene with Cylinder", s, [0, 0, 4], [0, 0, -1],
                  dict(hit=True, geom_id=0, distance=3.0, normal=[0, 0, 1])))
    s = W.SceneSpec()
    s.add_cylinders(np.array([[0.0, 0, -2]]), np.array([2.0]), np.array([2.0]), np.array([2.0]), I)
    s.add_spheres(np.array([[0.0, 0, 3]]), np.array([2.0]))
    cases.append(("Scene with 2 different primitives", s, [0, 0, 7], [0, 0, -1],
                  dict(hit=True, geom_id=1, prim_id=0, distance=2.0, normal=[0, 0, 1])))
    return cases


def spec_json(spec):
    d = {"order": spec.order}
    for k in spec.order:
        d[k] = {n: np.asarray(a).tolist() for n, a in getattr(spec, k).items()}
    return d


def make_kats(ref_root):
    runner = os.path.join(ROOT, "oracle", "_ref", "kat_runner")
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "kat.jsonl")
        r = subprocess.run([runner, path], capture_output=True, text=True)
        summary = json.loads(r.stdout.splitlines()[0])
        recs = [json.loads(l) for l in open(path)]
    assert summary["failed"] == 0, r.stdout
    for rec in recs:
        if rec["check"] in ("intersect_primitive", "traverse"):
            assert rec["direction_exact"], rec["case"]
            spec = spec_of(rec)
            ref = RefScene(spec)
            out = ref.intersect(np.array([rec["origin"]]), np.array([rec["direction"]]),
                                np.array([rec["tmin"]]), np.array([rec["tmax"]]))
            rec["scene_result"] = result_dict(out)
    scenes = []
    for name, spec, o, d, exp in scene_cases():
        out = RefScene(spec).intersect(np.array([o], float), np.array([d], float))
        scenes.append({"case": name, "check": "scene", "scene": spec_json(spec), "origin": o,
                       "direction": d, "tmin": 0.0, "tmax": DBL_MAX, "expected": exp,
                       "reference": result_dict(out)})
    return {"summary": summary, "source": "test/ of the reference via oracle/_ref/kat_runner",
            "records": recs + scenes}


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def make_configs():
    out = {}
    wl = W.icosphere_pinhole()
    idx = np.arange(0, wl.rays.n, 61)  # 4,298 rays spread over the image
    res = RefScene(wl.scene).intersect(wl.rays.origins[idx], wl.rays.directions[idx],
                                       wl.rays.tmin[idx], wl.rays.tmax[idx])
    out.update({f"icosphere_pinhole_{k}": res[k] for k in ("t", "uv", "normal", "prim", "geom", "hit")})
    out["icosphere_pinhole_idx"] = idx
    out["icosphere_pinhole_digest"] = np.frombuffer(bytes.fromhex(digest(
        wl.scene.mesh["vertices"], wl.scene.mesh["faces"], wl.rays.origins, wl.rays.directions)), np.uint8)
    wl = W.mixed_primitives()
    idx = np.arange(0, wl.rays.n, 128)  # 8,192 rays
    res = RefScene(wl.scene).intersect(wl.rays.origins[idx], wl.rays.directions[idx],
                                       wl.rays.tmin[idx], wl.rays.tmax[idx])
    out.update({f"mixed_primitives_{k}": res[k] for k in ("t", "uv", "normal", "prim", "geom", "hit")})
    out["mixed_primitives_idx"] = idx
    out["mixed_primitives_digest"] = np.frombuffer(bytes.fromhex(digest(
        wl.scene.spheres["centers"], wl.scene.cylinders["rotations"], wl.scene.planes["rotations"],
        wl.rays.origins, wl.rays.directions)), np.uint8)
    return out


def make_image_classes(ref_root):
    from PIL import Image

    im = np.array(Image.open(os.path.join(ref_root, "examples", "baseline", "scene_primitives.png")))
    red = (im[..., 0] == 255) & (im[..., 1] == 0)
    green = (im[..., 1] == 255) & (im[..., 0] == 0)
    assert not np.any(red & green)
    return {"shape": np.array(im.shape[:2]), "red": np.packbits(red), "green": np.packbits(green)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference",
                    default=os.path.normpath(os.path.join(HERE, "..", "..", "..", "reference")))
    a = ap.parse_args(argv)
    kats = make_kats(a.reference)
    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(kats, f, separators=(",", ":"))
    np.savez_compressed(os.path.join(HERE, "configs.npz"), **make_configs())
    np.savez_compressed(os.path.join(HERE, "scene_primitives_classes.npz"), **make_image_classes(a.reference))
    print("kats:", len(kats["records"]), "records;", kats["summary"])


if __name__ == "__main__":
    main()
