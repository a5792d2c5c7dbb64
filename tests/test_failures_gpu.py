"""Failure handling, made on the host (no GPU fault is involved):

* an allocation that fails on the k-th call (bzr_debug_fail_allocation, which reports the
  device as out of memory without allocating): the entry point that meets it returns
  BZR_ENOMEM, the scene stays usable, and once everything is closed the device holds no more
  memory than after a run without failures;
* a bounded wait that runs out: bzr_scene_check with a 1 ms limit on a long queued batch
  returns BZR_ETIMEOUT and a second check returns BZR_OK; a host-array call whose wait runs
  out returns BZR_ETIMEOUT, and the next call (which first waits for the late work on the
  staging buffers) gives the right results."""
import ctypes as C
import os

import numpy as np
import pytest

import blazert_b200 as B
from blazert_b200 import workloads as W
from tests.helpers import mismatches, to_numpy

pytestmark = pytest.mark.gpu


def _spec():
    rng = np.random.default_rng(5)
    return (W.SceneSpec().add_mesh(*W.icosphere(3))
            .add_spheres(rng.uniform(-1.5, 1.5, (200, 3)), rng.uniform(0.02, 0.1, 200)))


def _sequence(spec, rays, dev_rays, fail_at):
    """Every entry point that allocates, in turn, with the k-th allocation failing (0: none).
    Returns the status of each call ("ok" or the BZR_* code) and closes what it made."""
    import torch

    lib = B.library()
    lib.bzr_debug_fail_allocation.argtypes = [C.c_int64]
    lib.bzr_debug_fail_allocation(fail_at)
    status = []

    def call(fn):
        try:
            fn()
            status.append("ok")
            return True
        except B.BlazertError as e:
            status.append(e.code)
            return False

    o, d = rays
    od, dd, out = dev_rays
    scene = B.Scene()
    scene.add_mesh(*spec.mesh.values())
    scene.add_spheres(*spec.spheres.values())
    if not call(lambda: scene.commit(gpu_build=True)):
        assert call(lambda: scene.commit(gpu_build=True))  # usable after the failure
    call(lambda: scene.tune(sort=True, sort_min_rays=0))
    call(lambda: scene.intersectN(od, dd, out=out))  # device arrays: the sort's scratch
    call(lambda: torch.cuda.synchronize())
    call(lambda: scene.intersectN(od, dd, out={k: v for k, v in out.items() if k != "t"}))
    call(lambda: torch.cuda.synchronize())
    call(lambda: scene.intersectN(o[:100], d[:100]))  # host arrays, latency path
    call(lambda: scene.intersectN(o, d))  # host arrays, pipeline
    call(lambda: scene.distance_to_surface("mesh", np.arange(64, dtype=np.uint32) % 1280, o[:64]))
    call(lambda: scene.closest_surface(o[:4096]))
    call(lambda: scene.work_counts(o[:1000], d[:1000]))
    fwd = {}
    if call(lambda: fwd.update(scene.intersectN(od, dd))):
        call(lambda: scene.adjoint(od, dd, fwd, grad_t=torch.ones_like(fwd["t"])))
        call(lambda: torch.cuda.synchronize())
    batch = None

    def make_batch():
        nonlocal batch
        batch = B.Batch([scene])
    if call(make_batch):
        ts = torch.zeros(2, dtype=torch.int64, device=od.device)
        call(lambda: batch.intersect([0, od.shape[0]], od, dd, out=out, timestamps=ts))
        call(lambda: torch.cuda.synchronize())
        batch.close()
    scene.check()
    scene.close()
    lib.bzr_debug_fail_allocation(0)
    return status


def test_allocation_failures_report_enomem_and_leak_nothing():
    import torch

    dev = torch.device("cuda", 0)
    spec = _spec()
    rng = np.random.default_rng(6)
    n = 300_000
    o = rng.uniform(-3.0, 3.0, (n, 3))
    d = rng.normal(size=(n, 3))
    od, dd = torch.from_numpy(o).to(dev), torch.from_numpy(d).to(dev)
    f64 = torch.float64
    out = dict(t=torch.empty(n, dtype=f64, device=dev), uv=torch.empty((n, 2), dtype=f64, device=dev),
               normal=torch.empty((n, 3), dtype=f64, device=dev),
               prim=torch.empty(n, dtype=torch.int32, device=dev),
               geom=torch.empty(n, dtype=torch.int32, device=dev),
               hit=torch.empty(n, dtype=torch.uint8, device=dev))
    # a run without failures warms every cache (the device builder's workspace, torch's
    # allocator, the CUDA context) before the device's free memory is taken
    clean = _sequence(spec, (o, d), (od, dd, out), 0)
    assert all(s == "ok" for s in clean), clean
    _sequence(spec, (o, d), (od, dd, out), 0)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    # k = 1, 2, ... until three runs in a row meet no failure (k beyond the sequence's
    # allocations; an allocation with a fallback, such as the device builder's workspace, does
    # not fail its call)
    k, fired, clean_runs = 1, 0, 0
    while clean_runs < 3:
        status = _sequence(spec, (o, d), (od, dd, out), k)
        failed = [s for s in status if s != "ok"]
        assert all(s == B.ENOMEM for s in failed), (k, status)
        assert len(failed) <= 1, (k, status)
        fired += len(failed)
        clean_runs = 0 if failed else clean_runs + 1
        k += 1
        assert k < 200
    assert fired >= 10  # every allocating entry point met a failure once
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(dev)[0]
    assert free1 >= free0 - (4 << 20), (free0, free1)


def test_bounded_waits_time_out_and_recover():
    import torch

    dev = torch.device("cuda", 0)
    wl = W.mixed_primitives(n_rays=4_000_000, seed=31)
    R = wl.rays
    scene = B.Scene()
    for kind in wl.scene.order:
        getattr(scene, "add_" + kind)(*getattr(wl.scene, kind).values())
    scene.commit()
    od, dd = torch.from_numpy(R.origins).to(dev), torch.from_numpy(R.directions).to(dev)
    ref = to_numpy(scene.intersectN(od, dd))
    torch.cuda.synchronize()
    stream = torch.cuda.Stream(dev)
    out = scene.intersectN(od, dd, stream=stream)
    stream.synchronize()
    done = torch.cuda.Event()
    for _ in range(32):  # a few hundred milliseconds of queued work
        scene.intersectN(od, dd, out=out, stream=stream)
    done.record(stream)
    with pytest.raises(B.BlazertError) as e:
        scene.check(stream=stream.cuda_stream, timeout_ms=1)
    assert e.value.code == B.ETIMEOUT
    assert not done.query()  # the work was still queued when the wait ran out
    assert scene.check(stream=stream.cuda_stream, timeout_ms=60000) == 0
    # pinned host arrays (copies from pageable memory would return only once done): the call's
    # own wait runs out while its copies and kernels are queued
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    ho, hd = pin(R.origins), pin(R.directions)
    hout = dict(t=pin(np.empty(R.n)), uv=pin(np.empty((R.n, 2))), normal=pin(np.empty((R.n, 3))),
                prim=pin(np.empty(R.n, np.uint32)), geom=pin(np.empty(R.n, np.uint32)),
                hit=pin(np.empty(R.n, np.uint8)))
    os.environ["BZR_TIMEOUT_MS"] = "1"
    try:
        with pytest.raises(B.BlazertError) as e:
            scene.intersectN(ho, hd, out=hout)
        assert e.value.code == B.ETIMEOUT
    finally:
        del os.environ["BZR_TIMEOUT_MS"]
    got = scene.intersectN(ho, hd, out=hout)
    for k in ("prim", "geom"):
        ref[k] = ref[k].view(np.uint32)
    assert mismatches(got, ref) == []
    scene.close()
