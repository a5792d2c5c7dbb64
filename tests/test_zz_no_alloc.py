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


@pytest.mark.parametrize("mode", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", ["mixed_primitives", "heightfield"])
def test_noalloc_modes_and_kinds_allocate_nothing(name, mode):
    """Both modes, on a scene of several kinds and on a single-kind mesh scene: the results
    equal bzr_intersectN's bit for bit on two calls in a row, no allocation of this library is
    made (with the allocation-failure hook armed on the next allocation the calls still
    succeed), and the device's free memory does not change."""
    import torch

    wl = W.mixed_primitives(n_rays=200_000, seed=22) if name == "mixed_primitives" else \
        W.heightfield(n_rays=200_000, grid=256)
    R = wl.rays
    scene = product_scene(wl.scene)
    dev = torch.device("cuda", 0)
    o, d = torch.from_numpy(R.origins).to(dev), torch.from_numpy(R.directions).to(dev)
    tmin, tmax = torch.from_numpy(R.tmin).to(dev), torch.from_numpy(R.tmax).to(dev)
    ref = to_numpy(scene.intersectN(o, d, tmin, tmax, mode=("fp64", "mixed")[mode]))
    for k in ("prim", "geom"):
        ref[k] = ref[k].view(np.uint32)
    lib = B.library()
    lib.bzr_debug_fail_allocation.argtypes = [C.c_int64]
    stream = torch.cuda.current_stream(dev).cuda_stream
    n = R.n
    f64 = torch.float64
    out = dict(t=torch.empty(n, dtype=f64, device=dev), uv=torch.empty((n, 2), dtype=f64, device=dev),
               normal=torch.empty((n, 3), dtype=f64, device=dev),
               prim=torch.empty(n, dtype=torch.int32, device=dev),
               geom=torch.empty(n, dtype=torch.int32, device=dev),
               hit=torch.empty(n, dtype=torch.uint8, device=dev))
    lib.bzr_intersectN_noalloc.argtypes = [C.c_void_p, C.c_size_t] + [C.c_void_p] * 10 + \
        [C.c_int, C.c_void_p]
    ptr = lambda a: C.c_void_p(a.data_ptr())

    def call():
        return lib.bzr_intersectN_noalloc(scene._h, n, ptr(o), ptr(d), ptr(tmin), ptr(tmax),
                                          ptr(out["t"]), ptr(out["uv"]), ptr(out["normal"]),
                                          ptr(out["prim"]), ptr(out["geom"]), ptr(out["hit"]),
                                          mode, C.c_void_p(stream))

    assert call() == 0  # the first call on the device looks up the scratch's address
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    for _ in range(2):
        for v in out.values():
            v.fill_(7)
        lib.bzr_debug_fail_allocation(1)
        rc = call()
        lib.bzr_debug_fail_allocation(0)
        assert rc == 0, lib.bzr_last_error_string().decode()
        torch.cuda.synchronize()
        assert mismatches(out, ref) == []
    assert torch.cuda.mem_get_info(dev)[0] == free0
    assert scene.check() == 0
    scene.close()


def test_noalloc_rejects_host_arrays():
    """Host arrays are refused with BZR_EINVAL (the entry point stages nothing)."""
    wl = W.mixed_primitives(n_rays=1000, seed=23)
    R = wl.rays
    scene = product_scene(wl.scene)
    lib = B.library()
    lib.bzr_intersectN_noalloc.argtypes = [C.c_void_p, C.c_size_t] + [C.c_void_p] * 10 + \
        [C.c_int, C.c_void_p]
    t = np.empty(R.n)
    hp = lambda a: C.c_void_p(a.ctypes.data)
    rc = lib.bzr_intersectN_noalloc(scene._h, R.n, hp(R.origins), hp(R.directions), None, None,
                                    hp(t), None, None, None, None, None, 0, None)
    assert rc == B.EINVAL
    assert "device arrays" in lib.bzr_last_error_string().decode()
    scene.close()
