"""bzr_intersectN_noalloc, the entry point for callers that cannot allocate device memory while
they trace (a plugin inside a host application's frame loop, a service with a fixed memory
budget): called through the C-ABI twice in a row, its results must equal bzr_intersectN's bit
for bit.  The file sorts last so that a run stopping at the first failure has run the rest."""
import ctypes as C

import numpy as np
import pytest

import blazert_b200 as B
from blazert_b200 import workloads as W
from tests.helpers import mismatches, product_scene, to_numpy

pytestmark = pytest.mark.gpu


def _call(lib, scene, n, o, d, tmin, tmax, out, stream):
    ptr = lambda a: None if a is None else C.c_void_p(a.data_ptr())
    lib.bzr_intersectN_noalloc.argtypes = [C.c_void_p, C.c_size_t] + [C.c_void_p] * 10 + \
        [C.c_int, C.c_void_p]
    return lib.bzr_intersectN_noalloc(scene._h, n, ptr(o), ptr(d), ptr(tmin), ptr(tmax),
                                      ptr(out.get("t")), ptr(out.get("uv")), ptr(out.get("normal")),
                                      ptr(out.get("prim")), ptr(out.get("geom")), ptr(out.get("hit")),
                                      0, C.c_void_p(stream))


def test_noalloc_entry_matches_intersectN_twice():
    import torch

    wl = W.mixed_primitives(n_rays=300_000, seed=21)
    R = wl.rays
    scene = product_scene(wl.scene)
    dev = torch.device("cuda", 0)
    o, d = torch.from_numpy(R.origins).to(dev), torch.from_numpy(R.directions).to(dev)
    tmin, tmax = torch.from_numpy(R.tmin).to(dev), torch.from_numpy(R.tmax).to(dev)
    ref = to_numpy(scene.intersectN(o, d, tmin, tmax))
    for k in ("prim", "geom"):  # ids are unsigned; torch holds them as int32
        ref[k] = ref[k].view(np.uint32)
    lib = B.library()
    stream = torch.cuda.current_stream(dev).cuda_stream
    n = R.n

    def fresh():
        f64 = torch.float64
        return dict(t=torch.full((n,), -1.0, dtype=f64, device=dev),
                    uv=torch.full((n, 2), -1.0, dtype=f64, device=dev),
                    normal=torch.full((n, 3), -1.0, dtype=f64, device=dev),
                    prim=torch.full((n,), 7, dtype=torch.int32, device=dev),
                    geom=torch.full((n,), 7, dtype=torch.int32, device=dev),
                    hit=torch.full((n,), 3, dtype=torch.uint8, device=dev))

    for _ in range(2):  # the shared scratch keeps the previous call's contents
        out = fresh()
        assert _call(lib, scene, n, o, d, tmin, tmax, out, stream) == 0
        torch.cuda.synchronize()
        assert mismatches(out, ref) == []
    # without distances the passes carry the closest distance in the static scratch
    out = fresh()
    out.pop("t")
    assert _call(lib, scene, n, o, d, tmin, tmax, out, stream) == 0
    torch.cuda.synchronize()
    got = to_numpy(out)
    for k in ("prim", "geom", "hit"):
        assert np.array_equal(got[k].view(ref[k].dtype), ref[k]), k
    assert scene.check() == 0
    # batches above the stated maximum are rejected, not truncated
    big = 1 << 20 | 1
    ob = torch.zeros((big, 3), dtype=torch.float64, device=dev)
    rc = _call(lib, scene, big, ob, ob, None, None, dict(hit=torch.zeros(big, dtype=torch.uint8, device=dev)), stream)
    assert rc == B.EINVAL
    assert "1,048,576" in lib.bzr_last_error_string().decode()
