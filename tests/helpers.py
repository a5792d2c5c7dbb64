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
