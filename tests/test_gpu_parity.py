"""CUDA path vs the CPU oracle, bit for bit (prim_id, geom_id, hit flag, t, uv, normal).

The oracle is the C restatement of the reference (oracle/bzr_oracle.c), itself pinned to the
reference's own code in test_oracle_pin.py.  Inputs are the seeded synthetic workloads at full
size where the oracle finishes in seconds."""
import numpy as np
import pytest

from blazert_b200 import workloads as W
from oracle.oracle import Oracle
from tests.helpers import mismatches, product_scene

pytestmark = pytest.mark.gpu


def _run_both(wl, mode="fp64"):
    import torch

    R = wl.rays
    ref = Oracle(wl.scene).intersect(R.origins, R.directions, R.tmin, R.tmax)
    s = product_scene(wl.scene)
    dev = torch.device("cuda", 0)
    out_dev = s.intersectN(torch.from_numpy(R.origins).to(dev), torch.from_numpy(R.directions).to(dev),
                           None if R.tmin is None else torch.from_numpy(R.tmin).to(dev),
                           None if R.tmax is None else torch.from_numpy(R.tmax).to(dev), mode=mode)
    torch.cuda.synchronize()
    s.check()
    out_host = s.intersectN(R.origins, R.directions, R.tmin, R.tmax, mode=mode)
    return ref, out_dev, out_host


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["icosphere_pinhole", "mixed_primitives"])
def test_workload_bit_exact(name, mode):
    wl = W.WORKLOADS[name]()
    ref, out_dev, out_host = _run_both(wl, mode)
    assert ref["hit"].sum() > 0
    assert mismatches(out_dev, ref) == []
    assert mismatches(out_host, ref) == []


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_four_kinds_merge(mode):
    """All four kinds overlapping in space, so that every rule of the merge across kind passes
    (triangles first, strict '<' for later kinds, misses) decides some rays; device arrays and
    host arrays (in chunks) both equal the oracle."""
    wl = W.mixed_primitives(n_rays=400_000, n_spheres=2000, n_cylinders=400, n_planes=60, seed=31)
    v, f = W.icosphere(3)
    spec = W.SceneSpec().add_mesh(v * 60.0, f)
    for k in wl.scene.order:
        getattr(spec, "add_" + k)(*getattr(wl.scene, k).values())
    wl4 = W.Workload("four_kinds", spec, wl.rays, {})
    ref, out_dev, out_host = _run_both(wl4, mode)
    assert len(set(ref["geom"][ref["hit"] == 1].tolist())) == 4
    assert mismatches(out_dev, ref) == []
    assert mismatches(out_host, ref) == []


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
@pytest.mark.parametrize("max_depth", [62, 100])
def test_deep_tree_stack_storage(mode, max_depth):
    """150 spheres at x = 8^i (up to 3.6e134) with leaves of one sphere build a chain-like tree
    of depth 70 when max_tree_depth allows it.  Then the traversal stack (depth + 2 entries)
    exceeds the kernels' 64-entry thread-local stack and lives in shared memory; capped at
    depth 62 it fits the local stack.  Both must match the oracle built with the same
    options."""
    import torch

    import blazert_b200 as B

    n = 150
    c = np.zeros((n, 3))
    c[:, 0] = 8.0 ** np.arange(n)
    c[:, 1] = np.linspace(-0.05, 0.05, n)
    spec = W.SceneSpec().add_spheres(c, np.full(n, 0.1))
    rng = np.random.Generator(np.random.PCG64(71))
    k = rng.integers(0, n, 4096)
    o = np.stack([c[k, 0] - 1.0, rng.uniform(-0.2, 0.2, 4096), rng.uniform(-0.2, 0.2, 4096)], 1)
    d = np.stack([np.ones(4096), rng.uniform(-0.05, 0.05, 4096), rng.uniform(-0.05, 0.05, 4096)], 1)
    opts = B.BuildOptions(min_leaf_primitives=1, max_tree_depth=max_depth)
    s = product_scene(spec, opts)
    depth = s.stats("spheres")["max_depth"]
    assert (depth + 2 > 64) == (max_depth == 100), depth
    ref = Oracle(spec, min_leaf=1, max_depth=max_depth).intersect(o, d)
    assert ref["hit"].sum() > 500
    dev = torch.device("cuda", 0)
    out = s.intersectN(torch.from_numpy(o).to(dev), torch.from_numpy(d).to(dev), mode=mode)
    torch.cuda.synchronize()
    assert s.check() == 0
    assert mismatches(out, ref) == []


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["icosphere_pinhole", "mixed_primitives"])
def test_any_hit_bit_exact(name, mode):
    """Ray::AnyHit::yes for the whole batch (BZR_RAY_ANY_HIT): device and host arrays against
    the oracle's any-hit traversal (pinned to the reference in test_oracle_pin.py)."""
    import torch

    wl = W.WORKLOADS[name]()
    R = wl.rays
    ref = Oracle(wl.scene).intersect(R.origins, R.directions, R.tmin, R.tmax, any_hit=True)
    s = product_scene(wl.scene)
    dev = torch.device("cuda", 0)
    out_dev = s.intersectN(torch.from_numpy(R.origins).to(dev),
                           torch.from_numpy(R.directions).to(dev),
                           torch.from_numpy(R.tmin).to(dev), torch.from_numpy(R.tmax).to(dev),
                           mode=mode, any_hit=True)
    torch.cuda.synchronize()
    assert s.check() == 0
    out_host = s.intersectN(R.origins, R.directions, R.tmin, R.tmax, mode=mode, any_hit=True)
    assert mismatches(out_dev, ref) == []
    assert mismatches(out_host, ref) == []


def test_cpp_facade_runs_on_gpu(tmp_path):
    """The C++ facade end to end: reference-style code commits a four-kind scene and traces a
    closest-hit and an any-hit (shadow) ray through intersect1."""
    import os
    import subprocess

    from tests.test_capi import FACADE_APP, ROOT

    src = tmp_path / "app.cpp"
    src.write_text(FACADE_APP)
    exe = tmp_path / "app"
    lib = os.path.join(ROOT, "blazert_b200", "_lib")
    subprocess.run([os.environ.get("BZR_CXX", "g++"), "-std=c++17", "-O1", "-I",
                    os.path.join(ROOT, "include"), str(src), "-L", lib, "-lblazert_b200",
                    f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), "gpu"], check=True, capture_output=True, text=True)
    hit, geom, prim, t, hit2 = r.stdout.split()
    # the ray from (0.2, 0.2, 5) down -z meets the triangle at z = 2 first (t = 3), then sphere 0
    assert (hit, geom, prim, float(t), hit2) == ("1", "0", "0", 3.0, "1")


def test_embree_facade_runs_on_gpu(tmp_path):
    """EmbreeScene<float> and <double> (the reference's Embree-backend API) trace through the
    GPU path; the double scene's distance query, save and load work from C++."""
    import subprocess

    from tests.test_capi import EMBREE_APP, _compile

    exe = _compile(EMBREE_APP, tmp_path, "embree_app")
    r = subprocess.run([str(exe), str(tmp_path / "s.bzrscene")], check=True, capture_output=True,
                       text=True)
    f = r.stdout.split()
    # the ray from (3, 0, 5) down -z meets sphere 1 (centre (3, 0, 0), radius 0.5) at t = 4.5
    assert f[0] == "1" and f[1] == "1" and float(f[2]) == 4.5
    assert f[3] == "1" and f[4] == "1" and float(f[5]) == 4.5
    assert float(f[6]) == 2.0 and float(f[7]) == 2.5
    assert f[8] == "1" and float(f[9]) == 4.5
    assert f[10] == "1" and float(f[11]) == 4.0  # Scene<float>: unit sphere from z = 5


def test_intersect1_matches_batch():
    import blazert_b200 as B

    wl = W.mixed_primitives(n_rays=64, seed=5)
    s = product_scene(wl.scene)
    R = wl.rays
    ref = Oracle(wl.scene).intersect(R.origins, R.directions)
    for i in range(R.n):
        rh = B.RayHit()
        hit = B.intersect1(s, B.Ray(R.origins[i], R.directions[i]), rh)
        assert hit == bool(ref["hit"][i])
        assert rh.prim_id == ref["prim"][i] and rh.geom_id == ref["geom"][i]
        assert np.float64(rh.hit_distance).view(np.uint64) == ref["t"][i].view(np.uint64)


def test_tuning_changes_speed_not_results():
    """Every tuning knob (coherence sort, threads per block, stack storage, rays per warp
    fetch) and the autotuner's choice give the oracle's results."""
    import torch

    from blazert_b200.autotune import autotune

    wl = W.mixed_primitives(n_rays=300_000, seed=8)
    R = wl.rays
    ref = Oracle(wl.scene).intersect(R.origins, R.directions)
    s = product_scene(wl.scene)
    dev = torch.device("cuda", 0)
    o, d = torch.from_numpy(R.origins).to(dev), torch.from_numpy(R.directions).to(dev)
    configs = [dict(sort=True), dict(sort=False), dict(threads=64), dict(threads=256),
               dict(shared_stack=True), dict(shared_stack=True, threads=256), dict(chunk=0),
               dict(chunk=64), dict(chunk=128), dict(threads=128, shared_stack=False, chunk=32)]
    for cfg in configs:
        s.tune(sort_min_rays=0, **cfg)
        for mode in ("fp64", "mixed"):
            out = s.intersectN(o, d, mode=mode)
            torch.cuda.synchronize()
            assert s.check() == 0
            assert mismatches(out, ref) == [], (cfg, mode)
    res = autotune(s, o, d, sample=100_000)
    assert set(res["choice"]) == {"sort", "threads", "shared_stack", "chunk", "top_nodes"}
    out = s.intersectN(o, d)
    torch.cuda.synchronize()
    assert mismatches(out, ref) == []


def test_host_pipeline_knobs_change_speed_not_results():
    """Host-array calls with every pipeline shape (chunk count and size, edge chunks, grid
    share per chunk) and the host autotuner's choice give the oracle's results."""
    from blazert_b200.autotune import autotune_host

    wl = W.mixed_primitives(n_rays=700_000, seed=10)
    R = wl.rays
    ref = Oracle(wl.scene).intersect(R.origins, R.directions, R.tmin, R.tmax)
    s = product_scene(wl.scene)
    configs = [dict(host_chunks=1), dict(host_chunks=3, host_min_chunk=1024),
               dict(host_chunks=32, host_min_chunk=1024), dict(host_edge=50_000),
               dict(host_edge=1 << 20), dict(host_grid_div=2), dict(host_grid_div=8, host_chunks=12),
               dict(host_chunks=8, host_min_chunk=1 << 17, host_edge=0, host_grid_div=1)]
    for cfg in configs:
        s.tune(**cfg)
        out = s.intersectN(R.origins, R.directions, R.tmin, R.tmax)
        assert mismatches(out, ref) == [], cfg
    with pytest.raises(Exception):
        s.tune(host_chunks=33)
    with pytest.raises(Exception):
        s.tune(host_grid_div=0)
    res = autotune_host(s, R.origins, R.directions, R.tmin, R.tmax, reps=1, sweeps=1)
    assert set(res["choice"]) == {"host_min_chunk", "host_chunks", "host_grid_div", "host_edge"}
    assert mismatches(s.intersectN(R.origins, R.directions, R.tmin, R.tmax), ref) == []


@pytest.fixture(scope="module")
def heightfield_ref():
    wl = W.heightfield()
    R = wl.rays
    return wl, Oracle(wl.scene).intersect(R.origins, R.directions, R.tmin, R.tmax)


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_heightfield_full_size(mode, heightfield_ref):
    """2,093,058-triangle heightfield, 8,388,608 secondary rays, against the oracle."""
    import torch

    wl, ref = heightfield_ref
    R = wl.rays
    s = product_scene(wl.scene)
    dev = torch.device("cuda", 0)
    out = s.intersectN(torch.from_numpy(R.origins).to(dev), torch.from_numpy(R.directions).to(dev),
                       torch.from_numpy(R.tmin).to(dev), torch.from_numpy(R.tmax).to(dev), mode=mode)
    torch.cuda.synchronize()
    s.check()
    assert mismatches(out, ref) == []


def test_small_host_batches():
    """Host-array batches of up to 4,096 rays take the latency path (one packed copy each way,
    a grid sized to the batch): every output subset, with and without tmin / tmax, at the
    boundary sizes, against the oracle."""
    wl = W.mixed_primitives(n_rays=5000, seed=13)
    R = wl.rays
    s = product_scene(wl.scene)
    ora = Oracle(wl.scene)
    for n in (1, 2, 31, 4095, 4096, 4097):
        o, d = R.origins[:n], R.directions[:n]
        tmin = np.where(np.arange(n) % 3 == 0, 0.5, 0.0)
        tmax = np.where(np.arange(n) % 5 == 0, 60.0, np.inf)
        for lo, hi in ((None, None), (tmin, tmax)):
            ref = ora.intersect(o, d, lo, hi)
            assert mismatches(s.intersectN(o, d, lo, hi), ref) == [], (n, lo is None)
    # partial outputs: only the keys given are written
    import ctypes as C

    n = 100
    o, d = np.ascontiguousarray(R.origins[:n]), np.ascontiguousarray(R.directions[:n])
    ref = ora.intersect(o, d)
    t = np.full(n, -1.0)
    prim = np.zeros(n, np.uint32)
    lib = s._lib
    rc = lib.bzr_intersectN(s._h, n, o.ctypes.data, d.ctypes.data, None, None, t.ctypes.data,
                            None, None, prim.ctypes.data, None, None, 0, None)
    assert rc == 0
    hit = ref["hit"].astype(bool)
    assert np.array_equal(prim[hit], ref["prim"][hit])
    assert np.array_equal(t.view(np.uint64), np.asarray(ref["t"]).view(np.uint64))


def test_mixed_defers_uncovered_rays():
    """Rays the FP32 walk does not cover (zero and tiny direction components, far origins),
    mixed among ordinary rays on a scene of all four kinds: the mixed passes hand them to their
    FP64 passes, and every form of the call equals the oracle -- device arrays, host arrays (the
    latency path and the chunked pipeline), a sorted batch, shared-memory stacks, any-hit rays,
    and the entry point without allocations, whose scratch carries the list."""
    import ctypes as C

    import torch

    import blazert_b200 as B
    from tests.helpers import uncovered_workload

    wl, cls = uncovered_workload()
    R = wl.rays
    orc = Oracle(wl.scene)
    ref = orc.intersect(R.origins, R.directions, R.tmin, R.tmax)
    ref_any = orc.intersect(R.origins, R.directions, R.tmin, R.tmax, any_hit=True)
    for c in range(1, 5):
        assert ref["hit"][cls == c].sum() > 100
    s = product_scene(wl.scene)
    dev = torch.device("cuda", 0)
    o, d = torch.from_numpy(R.origins).to(dev), torch.from_numpy(R.directions).to(dev)
    tmn, tmx = torch.from_numpy(R.tmin).to(dev), torch.from_numpy(R.tmax).to(dev)
    for cfg in (dict(sort=False), dict(sort=True, sort_min_rays=0), dict(shared_stack=True)):
        s.tune(**cfg)
        out = s.intersectN(o, d, tmn, tmx, mode="mixed")
        torch.cuda.synchronize()
        assert s.check() == 0
        assert mismatches(out, ref) == [], cfg
        out = s.intersectN(o, d, tmn, tmx, mode="mixed", any_hit=True)
        torch.cuda.synchronize()
        assert mismatches(out, ref_any) == [], cfg
    s.tune(sort=False)
    assert mismatches(s.intersectN(R.origins, R.directions, R.tmin, R.tmax, mode="mixed"), ref) == []
    few = {k: v[:500] for k, v in ref.items()}
    assert mismatches(s.intersectN(R.origins[:500], R.directions[:500], R.tmin[:500],
                                   R.tmax[:500], mode="mixed"), few) == []
    lib = B.library()
    lib.bzr_intersectN_noalloc.argtypes = [C.c_void_p, C.c_size_t] + [C.c_void_p] * 10 + \
        [C.c_int, C.c_void_p]
    n = R.n
    f64 = torch.float64
    got = dict(t=torch.empty(n, dtype=f64, device=dev), uv=torch.empty((n, 2), dtype=f64, device=dev),
               normal=torch.empty((n, 3), dtype=f64, device=dev),
               prim=torch.empty(n, dtype=torch.int32, device=dev),
               geom=torch.empty(n, dtype=torch.int32, device=dev),
               hit=torch.empty(n, dtype=torch.uint8, device=dev))
    ptr = lambda a: C.c_void_p(a.data_ptr())
    for _ in range(2):
        for v in got.values():
            v.fill_(7)
        rc = lib.bzr_intersectN_noalloc(s._h, n, ptr(o), ptr(d), ptr(tmn), ptr(tmx), ptr(got["t"]),
                                        ptr(got["uv"]), ptr(got["normal"]), ptr(got["prim"]),
                                        ptr(got["geom"]), ptr(got["hit"]), 1,
                                        C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        assert mismatches(got, ref) == []
    assert s.check() == 0
    s.close()
