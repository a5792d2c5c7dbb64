#!/usr/bin/env python3
"""Mrays/s of blazeRT closest-hit queries (intersect1 semantics) on B200: FP64 vs mixed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload heightfield] [--mode both|fp64|mixed]

Workload (default): the 2,093,058-triangle heightfield -- a 1024 x 1024 vertex grid over
[0, 1000]^2 with 6-octave value-noise fBm heights (amplitude 100) -- and 8,388,608 secondary
rays leaving the surface (area-weighted points offset 1e-6 along the normal, cosine-weighted
directions), float64, seeded.  A step is one intersectN over the whole batch.

  value      Mrays/s of the FP64 path over all ranks, rays resident in HBM, device time (CUDA
             events on the launching stream), the L2 flushed (256 MiB written) between timed
             steps.
  precision  the mixed FP32/FP64 path timed the same way on the same rays (--mode both, the
             default): its Mrays/s, its ratio to the FP64 path, hit mismatches and distance
             errors against the FP64 path's results, and its own e2e.
  e2e        the same metric through the public host API (Scene.intersectN with pinned host
             arrays): host->device copy of the rays, the kernel, device->host copy of all
             results, every step.
  roofline   the FP64 traversal kernel against two measured ceilings: algorithmic bytes (ray
             I/O 121 B + 64 B per box test + the primitive record per primitive test; counts
             from the counting kernel) against the L2 read bandwidth measured in the run
             (bound "l2"), and the compulsory bytes (ray I/O + the scene's device image once)
             against the HBM copy bandwidth (MEASURED_PEAKS.json).
  cpu_baseline  the reference's own intersect1 loop (its headers, release flags, OpenMP over
             all host cores) on a bounded sample of the same rays, rank 0 at N = 1; also on
             one core, with the host's CPU model.

Other forms: --workload mixed_primitives | icosphere_pinhole (same line), batched_icospheres
(batching), adjoint_scene (differentiation), distance_queries (the reference's per-primitive
distance_to_surface over 4M (primitive, point) pairs per kind, Mqueries/s) and closest_surface
(nearest surface over the scene for 1M points, Mqueries/s).

Multi-GPU: one process per GPU (torchrun); every rank holds the scene and traces its own batch
(weak scaling, no data-path collective); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

RAY_IO_BYTES = 24 + 24 + 8 + 8 + 8 + 16 + 24 + 4 + 4 + 1  # o, d, tmin, tmax | t, uv, n, ids, hit
# bytes a primitive test consumes: triangle = {i0, i1, i2, id} + three 24-byte vertex positions;
# the other kinds read their record and 4-byte id word
PRIM_RECORD_BYTES = {0: 16 + 3 * 24, 1: 32 + 4, 2: 112 + 4, 3: 128 + 4}
BOX_TEST_BYTES = 64
METRIC = "Mrays/s closest-hit on 1 B200: FP64 vs mixed FP32/FP64, same hits; vs CPU"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="heightfield")
    ap.add_argument("--mode", default="both", choices=["both", "fp64", "mixed"],
                    help="both: value = the FP64 path, precision = the mixed path on the same "
                         "rays")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--rays", type=int, default=0,
                    help="override the workload's ray count (smaller cases for profiling)")
    ap.add_argument("--any-hit", action="store_true",
                    help="every ray with Ray::AnyHit::yes (shadow rays)")
    ap.add_argument("--sort", default="auto", choices=["auto", "on", "off"],
                    help="coherence sort of each batch; auto = chosen by blazert_b200.autotune")
    return ap.parse_args(argv)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.dev)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# Rays of the bounded CPU samples (all host cores; one core), per workload: about 10 s and 5 s
# of the reference's ray loop.
CPU_SAMPLE_RAYS = {"heightfield": 1 << 20, "adjoint_scene": 1 << 20}
CPU_ONE_CORE_RAYS = {"heightfield": 1 << 16, "mixed_primitives": 1 << 16,
                     "icosphere_pinhole": 1 << 18, "adjoint_scene": 1 << 16,
                     "batched_icospheres": 1 << 12}


def cpu_baseline(workload, seconds, max_rays=0):
    """The reference's intersect1 loop on this host: all cores (the reported baseline) and one
    core (comparable with the reference's own single-thread plots), with the CPU model."""
    def run(threads, secs, rays):
        cmd = [sys.executable, "-m", "oracle.cpu_baseline", "--workload", workload,
               "--seconds", str(secs), "--threads", str(threads)]
        if rays:
            cmd += ["--max-rays", str(rays)]
        r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
        if r.returncode != 0:
            return {"error": r.stderr.strip()[-400:]}
        return json.loads(r.stdout.strip().splitlines()[-1])

    out = run(0, seconds, max_rays)
    if "error" not in out:
        one = run(1, seconds / 2, CPU_ONE_CORE_RAYS.get(workload, 1 << 16))
        out["one_core"] = {k: one.get(k) for k in ("value", "unit", "sample", "error") if k in one}
    return out


def config_of(args, wl, world, mode="fp64"):
    m = wl.meta
    return {"workload": args.workload, "rays_per_gpu": wl.rays.n,
            "scene": {k: v for k, v in m.items() if k != "seed"},
            "seed": m.get("seed"), "mode": mode,
            "modes_timed": ["fp64", "mixed"] if args.mode == "both" else [args.mode],
            "parallelism": f"replicated-scene x{world}",
            "rays": "any-hit (shadow)" if getattr(args, "any_hit", False) else "closest-hit",
            "l2": "flushed between timed steps (256 MiB write)"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from blazert_b200 import workloads as W
    from oracle.cpu_baseline import host_cpu
    from oracle.oracle import Oracle, RefScene
    threads = os.cpu_count() or 1
    if args.workload in W.DISTANCE_WORKLOADS:
        # the reference's distance functions on every host core; steps of the closest-surface
        # workload are bounded samples (the reference has no scene-level query: every point
        # is checked against every primitive)
        from oracle.cpu_baseline import measure_distance
        m = measure_distance(args.workload, seconds=0.0, threads=threads,
                             max_queries=0 if args.workload == "distance_queries" else 2048,
                             min_reps=args.warmup + args.steps)
        print(json.dumps({
            "metric": ("Mqueries/s distance_to_surface (per-primitive, bit-exact) on 1 B200"
                       if args.workload == "distance_queries" else
                       "Mqueries/s nearest surface over the scene (bit-exact) on 1 B200"),
            "value": m["value"], "unit": "Mqueries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * m["seconds_per_batch"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": args.workload,
                                                     "queries_per_step": m["queries"]},
            "impl": "reference",
            "cpu_baseline": {k: m[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": m["value"], "unit": "Mqueries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return 0
    wl = W.WORKLOADS[args.workload](**({"n_rays": args.rays} if args.rays else {}))
    kind = "reference" if RefScene.available("bench") else "port"
    sc = RefScene(wl.scene, flavour="bench") if kind == "reference" else Oracle(wl.scene)
    R = wl.rays

    def step():
        t0 = time.perf_counter()
        sc.intersect(R.origins, R.directions, R.tmin, R.tmax, nthreads=threads)
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    times = [step() for _ in range(args.steps)]
    total = sum(times)
    value = R.n * args.steps / total / 1e6
    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": config_of(args, wl, 1), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": kind,
                             "sample": f"{args.workload}: full batch of {R.n} rays per step",
                             **host_cpu()},
            "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_batched(args):
    """Batching form: 256 perturbed icospheres with uneven ray batches, one launch per kind,
    replayed from a CUDA graph; per-scene latency from the kernels' completion timestamps."""
    import numpy as np
    import torch

    import blazert_b200 as B
    from blazert_b200 import workloads as W

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scale = args.rays / 37_000_000 if args.rays else 1.0
    wls = W.batched_icospheres(seed=4 + rank, scale=scale)
    t0 = time.perf_counter()
    scenes = []
    for w in wls:
        sc = B.Scene()
        sc.add_mesh(*w.scene.mesh.values())
        sc.commit()
        scenes.append(sc)
    commit_s = time.perf_counter() - t0
    batch = B.Batch(scenes)
    offs = np.concatenate([[0], np.cumsum([w.rays.n for w in wls])]).astype(np.int64)
    tuning = None
    n = int(offs[-1])
    o = torch.from_numpy(np.concatenate([w.rays.origins for w in wls])).to(dev)
    d = torch.from_numpy(np.concatenate([w.rays.directions for w in wls])).to(dev)
    tmn = torch.zeros(n, dtype=torch.float64, device=dev)
    tmx = torch.full((n,), float("inf"), dtype=torch.float64, device=dev)
    ts = torch.zeros(len(wls) + 1, dtype=torch.int64, device=dev)
    f64 = torch.float64
    out = dict(t=torch.empty(n, dtype=f64, device=dev), uv=torch.empty((n, 2), dtype=f64, device=dev),
               normal=torch.empty((n, 3), dtype=f64, device=dev),
               prim=torch.empty(n, dtype=torch.int32, device=dev),
               geom=torch.empty(n, dtype=torch.int32, device=dev),
               hit=torch.empty(n, dtype=torch.uint8, device=dev))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    if args.sort == "auto":  # the batch kernels' launch shape, chosen on this batch
        from blazert_b200.autotune import autotune_batch
        tuning = autotune_batch(batch, offs, o, d, tmn, tmx, mode=args.mode, stream=stream)
    for i in range(args.warmup):
        flush.fill_(i & 0xFF)
        batch.intersect(offs, o, d, tmn, tmx, out=out, timestamps=ts, mode=args.mode, stream=stream)
    torch.cuda.synchronize(dev)
    batch.check()
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    lat = []
    for i in range(args.steps):
        flush.fill_((i + 1) & 0xFF)
        evs[i][0].record(stream)
        batch.intersect(offs, o, d, tmn, tmx, out=out, timestamps=ts, mode=args.mode, stream=stream)
        evs[i][1].record(stream)
        stream.synchronize()
        t = ts.cpu().numpy()
        lat.append((t[:-1] - t[-1]) / 1e6)  # ms per scene
    clocks = sampler.stop() if sampler else None
    batch.check()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = sum(step_ms)
    lat = np.concatenate(lat)
    value = world * n * args.steps / (total_ms / 1e3) / 1e6
    # compulsory HBM bytes of a step: every ray's I/O and every scene's FP64 device image once
    # (internal nodes, triangle index words and vertices)
    s_bytes = 0
    for sc, w in zip(scenes, wls):
        st = sc.build_statistics("mesh")
        s_bytes += 128 * st["branch_nodes"] + 16 * len(w.scene.mesh["faces"]) + \
            32 * len(w.scene.mesh["vertices"])
    hbm_peak, peak_src = load_peaks()
    mean_ms = statistics.mean(step_ms)
    hbm_achieved = (n * RAY_IO_BYTES + s_bytes) / (mean_ms / 1e3) / 1e9
    roofline = {"bound": "latency", "achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": hbm_achieved / hbm_peak, "traffic": None, "peak_source": peak_src,
                "what": "compulsory bytes (ray I/O 121 B per ray + each scene's device image "
                        "once) per step against the measured HBM copy bandwidth; the walk is "
                        "bound by dependent-load latency, far below it"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline("batched_icospheres", args.cpu_seconds)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": "batched_icospheres", "scenes": len(wls), "rays_per_gpu": n,
                       "scenes_per_level": {str(lv): sum(1 for w in wls if w.meta["level"] == lv)
                                            for lv in sorted({w.meta["level"] for w in wls})},
                       "mode": args.mode,
                       "graph": "CUDA graph replay", "l2": "flushed between timed steps"},
            "gpu_launches": args.steps * 2,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())},
            "roofline": roofline, "cpu_baseline": cpu,
            "clocks": clocks, "commit_seconds": commit_s, "tuning": tuning}), flush=True)
    return 0


def pcie_ceiling(in_bytes, out_bytes, dev, reps=3):
    """The copy ceiling of an end-to-end step: `in_bytes` from pinned host memory to the device
    and `out_bytes` back, on two streams at once (the two directions of PCIe run side by side),
    best of `reps`, timed by the wall clock around a synchronize like the e2e steps.  Returns
    milliseconds."""
    import torch

    hin = torch.empty(in_bytes, dtype=torch.uint8).pin_memory()
    hout = torch.empty(out_bytes, dtype=torch.uint8).pin_memory()
    din = torch.empty(in_bytes, dtype=torch.uint8, device=dev)
    dout = torch.empty(out_bytes, dtype=torch.uint8, device=dev)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    best = float("inf")
    for _ in range(reps + 1):  # the first round is a warm-up
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        with torch.cuda.stream(s_in):
            din.copy_(hin, non_blocking=True)
        with torch.cuda.stream(s_out):
            hout.copy_(dout, non_blocking=True)
        torch.cuda.synchronize(dev)
        best = min(best, (time.perf_counter() - t0) * 1e3)
    del hin, hout, din, dout
    return best


def l2_read_peak():
    """Measured L2 -> SM read bandwidth of the current GPU (GB/s): the probe library's
    ld.global.cg read of buffers that fit in L2, best over a few sizes (per-size figures too)."""
    import ctypes as C
    path = os.path.join(ROOT, "blazert_b200", "_lib", "libbzr_probe.so")
    if not os.path.exists(path):
        return None, {}
    lib = C.CDLL(path)
    lib.bzr_probe_read_gbs.argtypes = [C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.bzr_probe_read_gbs.restype = C.c_int
    per = {}
    for mb in (8, 16, 32, 48):
        g = C.c_double(0.0)
        if lib.bzr_probe_read_gbs(mb << 20, 40, 1, C.byref(g)) == 0:
            per[f"{mb}MiB"] = g.value
    return (max(per.values()) if per else None), per


def scene_bytes(scene, wl):
    """Bytes of the FP64 device image a launch needs at least once (S of the compulsory HBM
    ceiling): per kind 128 B per internal node plus the leaf-ordered primitive data (mesh:
    16 B per triangle and 32 B per vertex)."""
    total = 0
    rec = {"spheres": 32 + 4, "planes": 112 + 4, "cylinders": 128 + 4}
    for kind in wl.scene.order:
        st = scene.build_statistics(kind)
        total += 128 * st["branch_nodes"]
        if kind == "mesh":
            total += 16 * len(wl.scene.mesh["faces"]) + 32 * len(wl.scene.mesh["vertices"])
        else:
            total += rec[kind] * len(next(iter(getattr(wl.scene, kind).values())))
    return total


def time_steps(step, stream, flush, steps, warmup, dev, pg):
    """W untimed steps, then K steps each bracketed by CUDA events on `stream`, the L2 flushed
    (256 MiB written) before every step; barrier + synchronize on both sides of the timed
    region.  Returns the per-step times and their total, the max over ranks."""
    import torch

    from blazert_b200 import multi
    for i in range(warmup):
        flush.fill_(i & 0xFF)
        step()
    torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    for i in range(steps):
        flush.fill_((i + 1) & 0xFF)  # untimed: evicts the previous step's rays from L2
        evs[i][0].record(stream)
        step()
        evs[i][1].record(stream)
    torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = sum(step_ms)
    if pg:
        total_ms = multi.max_over_ranks(total_ms)
    return step_ms, total_ms


def run_ours(args):
    import numpy as np
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        pg = dist
    import blazert_b200 as B
    from blazert_b200 import multi
    from blazert_b200 import workloads as W

    modes = ["fp64", "mixed"] if args.mode == "both" else [args.mode]
    wl = W.WORKLOADS[args.workload](**({"n_rays": args.rays} if args.rays else {}))
    R = wl.rays
    if rank > 0:  # weak scaling: each rank traces its own full-size batch
        R = W.RayBatch(*multi.rank_batch(R.origins, R.directions, R.tmin, R.tmax, rank))
    scene = B.Scene()
    for kind in wl.scene.order:
        d = getattr(wl.scene, kind)
        getattr(scene, "add_" + kind)(*d.values())
    t0 = time.perf_counter()
    scene.commit()
    commit_s = time.perf_counter() - t0
    n = R.n
    o = torch.from_numpy(R.origins).to(dev)
    d = torch.from_numpy(R.directions).to(dev)
    tmn = torch.from_numpy(R.tmin).to(dev)
    tmx = torch.from_numpy(R.tmax).to(dev)
    f64 = torch.float64

    def outputs():
        return dict(t=torch.empty(n, dtype=f64, device=dev),
                    uv=torch.empty((n, 2), dtype=f64, device=dev),
                    normal=torch.empty((n, 3), dtype=f64, device=dev),
                    prim=torch.empty(n, dtype=torch.int32, device=dev),
                    geom=torch.empty(n, dtype=torch.int32, device=dev),
                    hit=torch.empty(n, dtype=torch.uint8, device=dev))

    outs = {m: outputs() for m in modes}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    l2_peak, l2_sizes = l2_read_peak()
    hbm_peak, peak_src = load_peaks()

    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    res = {}
    wall0 = time.perf_counter()
    for m in modes:
        tuning = None
        if args.sort == "auto":
            from blazert_b200.autotune import autotune
            tuning = autotune(scene, o, d, tmn, tmx, mode=m, stream=stream)
        else:
            scene.tune(sort=args.sort == "on")

        def step(m=m):
            scene.intersectN(o, d, tmn, tmx, mode=m, out=outs[m], stream=stream,
                             any_hit=args.any_hit)

        step_ms, total_ms = time_steps(step, stream, flush, args.steps, args.warmup, dev, pg)
        scene.check()
        res[m] = dict(step_ms=step_ms, total_ms=total_ms, tuning=tuning,
                      value=world * n * args.steps / (total_ms / 1e3) / 1e6)
    wall = time.perf_counter() - wall0
    clocks = sampler.stop() if sampler else None
    primary = modes[0]
    value, total_ms, step_ms = res[primary]["value"], res[primary]["total_ms"], res[primary]["step_ms"]
    out = outs[primary]
    hits = float(out["hit"].float().mean().item())

    precision = None
    if "mixed" in modes:  # the precision form's report: its results against the FP64 path's
        got = outs["mixed"]
        ref = outs["fp64"] if "fp64" in outs else scene.intersectN(
            o, d, tmn, tmx, mode="fp64", stream=stream, any_hit=args.any_hit)
        torch.cuda.synchronize(dev)
        same = (got["hit"] == ref["hit"]) & (got["prim"] == ref["prim"]) & \
            (got["geom"] == ref["geom"])
        both = (got["hit"] == 1) & (ref["hit"] == 1)
        rel = ((got["t"] - ref["t"]).abs() / ref["t"].abs().clamp_min(1e-300))[both]
        eq = lambda k: torch.equal(got[k].view(torch.int64), ref[k].view(torch.int64))
        precision = {
            "mode": "mixed", "value": res["mixed"]["value"], "unit": "Mrays/s",
            "ms_per_step": res["mixed"]["total_ms"] / args.steps,
            "vs_fp64": (res["mixed"]["value"] / res["fp64"]["value"]) if "fp64" in res else None,
            "against": "FP64 GPU path of the same run (bit-identical to the oracle in the "
                       "parity tests)",
            "hit_mismatches": int((~same).sum().item()),
            "t_max_rel_err": float(rel.max().item()) if rel.numel() else 0.0,
            "t_mean_rel_err": float(rel.mean().item()) if rel.numel() else 0.0,
            "t_uv_normal_bit_identical": bool(eq("t") and eq("uv") and eq("normal")),
            "tuning": res["mixed"]["tuning"],
            "step_ms_min_max": [min(res["mixed"]["step_ms"]), max(res["mixed"]["step_ms"])]}
    # one traversal kernel per primitive kind present, per step
    n_passes = sum(1 for k in wl.scene.order if len(next(iter(getattr(wl.scene, k).values()))))
    # kernels per call: one per kind present; in the mixed mode the triangle, sphere and plane
    # passes add the FP64 pass over the rays their FP32 test does not cover
    n_wide = sum(1 for k in wl.scene.order
                 if k != "cylinders" and len(next(iter(getattr(wl.scene, k).values()))))
    launches_per_call = {"fp64": n_passes, "mixed": n_passes + n_wide}

    # roofline of the primary path's traversal kernel.  Algorithmic bytes from the kernel's own
    # work counts (untimed counting run): ray I/O + 64 B per box test (half a 128-byte two-child
    # node) + the primitive record per primitive test.
    counts = scene.work_counts(o, d, tmn, tmx, stream=stream)
    alg_bytes = n * RAY_IO_BYTES + BOX_TEST_BYTES * sum(counts["box"]) + \
        sum(PRIM_RECORD_BYTES[k] * counts["prim"][k] for k in range(4))
    mean_ms = statistics.mean(step_ms)
    achieved = alg_bytes / (mean_ms / 1e3) / 1e9
    s_bytes = scene_bytes(scene, wl)
    hbm_need = n * RAY_IO_BYTES + s_bytes
    hbm_achieved = hbm_need / (mean_ms / 1e3) / 1e9
    traffic, traffic_src = None, None
    tf = os.path.join(ROOT, "profiles", f"trace_fp64_{args.workload}.json")
    if os.path.exists(tf) and not args.any_hit and primary == "fp64":
        with open(tf) as f:
            tj = json.load(f)
        traffic = tj.get("dram_bytes_per_launch")
        traffic_src = tj.get("source")
    frac_l2 = achieved / l2_peak if l2_peak else None
    roofline = {
        "bound": "l2", "achieved": achieved, "peak": l2_peak, "unit": "GB/s", "frac": frac_l2,
        "traffic": traffic, "traffic_source": traffic_src,
        "peak_source": "measured in this run (L2-resident ld.global.cg read, best of "
                       + ", ".join(f"{k}: {v:.0f}" for k, v in l2_sizes.items()) + " GB/s)",
        "alg_bytes_per_ray": alg_bytes / n,
        "box_tests_per_ray": [c / n for c in counts["box"]],
        "prim_tests_per_ray": [c / n for c in counts["prim"]],
        "ceilings": {
            "l2": {"achieved": achieved, "peak": l2_peak, "frac": frac_l2,
                   "what": "algorithmic traversal bytes (ray I/O + box tests + primitive "
                           "records) / kernel time, against the measured L2 read bandwidth"},
            "hbm_compulsory": {"achieved": hbm_achieved, "peak": hbm_peak, "frac":
                               hbm_achieved / hbm_peak, "peak_source": peak_src,
                               "bytes_per_ray": RAY_IO_BYTES + s_bytes / n,
                               "what": "(ray I/O 120 B + scene bytes S / rays R) per ray, "
                                       "against the measured HBM copy bandwidth"}},
        "binding": ("latency and SIMD divergence: neither byte ceiling is reached (see the "
                    "ncu summaries: long-scoreboard stalls, active lanes per warp)"
                    if (frac_l2 or 0) < 0.6 and hbm_achieved / hbm_peak < 0.6 else "bandwidth"),
        "note": ("work counts are the closest-hit traversal's; any-hit rays do less, so "
                 "achieved is an upper bound") if args.any_hit else None}

    e2e, e2e_mixed = None, None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        ho, hd, htmn, htmx = pin(R.origins), pin(R.directions), pin(R.tmin), pin(R.tmax)
        hout = dict(t=torch.empty(n, dtype=f64).pin_memory().numpy(),
                    uv=torch.empty((n, 2), dtype=f64).pin_memory().numpy(),
                    normal=torch.empty((n, 3), dtype=f64).pin_memory().numpy(),
                    prim=torch.empty(n, dtype=torch.int32).pin_memory().numpy().view(np.uint32),
                    geom=torch.empty(n, dtype=torch.int32).pin_memory().numpy().view(np.uint32),
                    hit=torch.empty(n, dtype=torch.uint8).pin_memory().numpy())
        def device_knobs(m):
            if res[m]["tuning"]:  # the device knobs this mode was timed with
                c = res[m]["tuning"]["choice"]
                scene.tune(sort=c["sort"], sort_min_rays=0 if c["sort"] else 1 << 16,
                           threads=c["threads"], shared_stack=c["shared_stack"], chunk=c["chunk"],
                           top_nodes=c.get("top_nodes", 0))

        host_tuning = None
        if args.sort == "auto" and not args.any_hit:
            from blazert_b200.autotune import autotune_host
            device_knobs(primary)
            host_tuning = autotune_host(scene, ho, hd, htmn, htmx, out=hout, mode=primary)
            host_tuning = {"choice": host_tuning["choice"], "best_ms": host_tuning["best_ms"]}

        def e2e_of(m):
            device_knobs(m)
            for _ in range(max(1, args.warmup)):
                scene.intersectN(ho, hd, htmn, htmx, mode=m, out=hout, any_hit=args.any_hit)
            if pg:
                pg.barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                scene.intersectN(ho, hd, htmn, htmx, mode=m, out=hout, any_hit=args.any_hit)
            el = time.perf_counter() - t0
            if pg:
                el = multi.max_over_ranks(el)
            r = {"value": world * n * args.steps / el / 1e6, "unit": "Mrays/s",
                 "h2d_bytes_per_step": n * (24 + 24 + 8 + 8),
                 "d2h_bytes_per_step": n * (8 + 16 + 24 + 4 + 4 + 1), "mode": m}
            if not np.array_equal(hout["prim"], outs[m]["prim"].cpu().numpy().view(np.uint32)):
                r["warning"] = "host-path results differ from the device path"
            return r

        e2e = e2e_of(primary)
        e2e["host_tuning"] = host_tuning
        # the step's own copies, alone: what the copy engines allow for these bytes
        copy_ms = pcie_ceiling(e2e["h2d_bytes_per_step"], e2e["d2h_bytes_per_step"], dev)
        copy_value = world * n / (copy_ms / 1e3) / 1e6
        e2e["ceiling"] = {"value": copy_value, "unit": "Mrays/s", "copy_ms": copy_ms,
                          "frac": e2e["value"] / copy_value,
                          "what": "the step's host<->device bytes copied alone, both directions "
                                  "at once from pinned memory (no kernels)"}
        if precision is not None and primary != "mixed":
            mixed_tuning = None
            if host_tuning is not None:  # the pipeline's knobs, chosen again for this mode
                from blazert_b200.autotune import autotune_host
                device_knobs("mixed")
                mixed_tuning = autotune_host(scene, ho, hd, htmn, htmx, out=hout, mode="mixed")
                mixed_tuning = {"choice": mixed_tuning["choice"],
                                "best_ms": mixed_tuning["best_ms"]}
            e2e_mixed = e2e_of("mixed")
            e2e_mixed["host_tuning"] = mixed_tuning
            precision["e2e"] = e2e_mixed

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.workload, args.cpu_seconds,
                           max_rays=CPU_SAMPLE_RAYS.get(args.workload, 0))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": config_of(args, wl, world, primary),
            "e2e": e2e, "gpu_launches": args.steps * sum(launches_per_call[m] for m in modes),
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks, "hit_fraction": hits,
            "precision": precision, "commit_seconds": commit_s, "wall_seconds_timed": wall,
            "tuning": res[primary]["tuning"], "step_ms_min_max": [min(step_ms), max(step_ms)],
        }
        print(json.dumps(line), flush=True)
    scene.close()
    if pg:
        pg.destroy_process_group()
    return 0


# bytes the adjoint reads and writes per ray hit: rays (48), forward record t/prim/geom/hit
# (17), dL/dt (8), dL/d(origin, direction) out (48), three vertices or one sphere (72) read and
# their gradient accumulated (72)
ADJOINT_BYTES_PER_RAY = 48 + 17 + 8 + 48 + 72 + 72


def run_adjoint(args):
    """Differentiation form: one step = the forward closest-hit pass over the batch, dL/dt of
    L = sum w_i t_i^2 (w ~ N(0, 1), misses contribute 0), and the adjoint kernels giving
    dL/d(vertices, sphere centres and radii, ray origins and directions).  Mrays/s of the whole
    step; the adjoint's own time is reported beside it."""
    import numpy as np
    import torch

    import blazert_b200 as B
    from blazert_b200 import multi
    from blazert_b200 import workloads as W

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    wl = W.adjoint_scene(**({"n_rays": args.rays} if args.rays else {}))
    R = wl.rays
    if rank > 0:
        R = W.RayBatch(*multi.rank_batch(R.origins, R.directions, R.tmin, R.tmax, rank))
    spec = wl.scene
    scene = B.Scene()
    for kind in spec.order:
        getattr(scene, "add_" + kind)(*getattr(spec, kind).values())
    scene.commit()
    n = R.n
    nv, ns = len(spec.mesh["vertices"]), len(spec.spheres["radii"])
    o = torch.from_numpy(R.origins).to(dev)
    d = torch.from_numpy(R.directions).to(dev)
    w = torch.from_numpy(np.asarray(wl.meta["weights"])[:n]).to(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step(ev=None):
        fwd = scene.intersectN(o, d, stream=stream)
        gt = torch.where(fwd["hit"].bool(), 2.0 * w * fwd["t"], torch.zeros_like(w))
        if ev is not None:
            ev.record(stream)
        return scene.adjoint(o, d, fwd, grad_t=gt, n_vertices=nv, n_spheres=ns, stream=stream)

    for i in range(args.warmup):
        flush.fill_(i & 0xFF)
        step()
    torch.cuda.synchronize(dev)
    scene.check()
    if pg:
        pg.barrier()
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    for i in range(args.steps):
        flush.fill_((i + 1) & 0xFF)
        evs[i][0].record(stream)
        step(evs[i][1])
        evs[i][2].record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop() if sampler else None
    scene.check()
    total_ms = sum(a.elapsed_time(c) for a, _, c in evs)
    adj_ms = sum(b.elapsed_time(c) for _, b, c in evs)
    if pg:
        total_ms = multi.max_over_ranks(total_ms)
        adj_ms = multi.max_over_ranks(adj_ms)
    value = world * n * args.steps / (total_ms / 1e3) / 1e6
    fwd = scene.intersectN(o, d, stream=stream)
    hit_frac = float(fwd["hit"].float().mean().item())
    counts = scene.work_counts(o, d, stream=stream)
    fwd_bytes = n * RAY_IO_BYTES + BOX_TEST_BYTES * sum(counts["box"]) + \
        sum(PRIM_RECORD_BYTES[k] * counts["prim"][k] for k in range(4))
    alg_bytes = fwd_bytes + hit_frac * n * ADJOINT_BYTES_PER_RAY
    achieved = alg_bytes / (total_ms / args.steps / 1e3) / 1e9
    peak, peak_src = load_peaks()

    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        ho, hd = pin(R.origins), pin(R.directions)
        hw = pin(np.asarray(wl.meta["weights"])[:n])
        host_out = {k: torch.empty(shape, dtype=torch.float64).pin_memory()
                    for k, shape in (("vertices", (nv, 3)), ("centers", (ns, 3)),
                                     ("radii", (ns,)), ("origins", (n, 3)),
                                     ("directions", (n, 3)))}

        def e2e_step():
            o.copy_(ho, non_blocking=True)
            d.copy_(hd, non_blocking=True)
            w.copy_(hw, non_blocking=True)
            g = step()
            for k, t in host_out.items():
                t.copy_(g[k], non_blocking=True)

        for _ in range(max(1, args.warmup)):
            e2e_step()
        torch.cuda.synchronize(dev)
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        torch.cuda.synchronize(dev)
        el = time.perf_counter() - t0
        if pg:
            el = multi.max_over_ranks(el)
        e2e = {"value": world * n * args.steps / el / 1e6, "unit": "Mrays/s",
               "h2d_bytes_per_step": n * (24 + 24 + 8),
               "d2h_bytes_per_step": 8 * (3 * nv + 3 * ns + ns + 6 * n)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference has no adjoint: its intersect1 loop over the same rays (the forward
        # pass only) is the CPU figure
        cpu = cpu_baseline("adjoint_scene", args.cpu_seconds,
                           max_rays=CPU_SAMPLE_RAYS.get("adjoint_scene", 0))
        cpu["what"] = "forward pass only (the reference has no adjoint)"
    if rank == 0:
        print(json.dumps({
            "metric": METRIC + " (forward + adjoint)", "value": value, "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": "adjoint_scene", "rays_per_gpu": n, "triangles": len(spec.mesh["faces"]),
                       "spheres": ns, "loss": "sum w t^2, w ~ N(0,1)",
                       "l2": "flushed between timed steps (256 MiB write)"},
            "adjoint_ms_per_step": adj_ms / args.steps, "hit_fraction": hit_frac,
            "e2e": e2e,
            "gpu_launches": args.steps * 4,  # two kind passes, the ray and face adjoint kernels
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_source": peak_src},
            "cpu_baseline": cpu, "clocks": clocks}), flush=True)
    if pg:
        pg.destroy_process_group()
    return 0


DIST_RECORD_BYTES = {"mesh": 16 + 3 * 24, "spheres": 32, "planes": 112, "cylinders": 128}


def run_distance(args):
    """Distance form.  distance_queries: one step = bzr_distance_to_surface over 4,194,304
    (primitive, point) pairs of each kind of the mixed-primitive scene (one launch per kind).
    closest_surface: one step = bzr_closest_surface over 1,048,576 points in the box of the
    differentiation scene (91,920 triangles, 500 spheres).  Mqueries/s, device time, the L2
    flushed between steps; e2e through Scene.distance_to_surface / closest_surface with pinned
    host arrays."""
    import numpy as np
    import torch

    import blazert_b200 as B
    from blazert_b200 import multi
    from blazert_b200 import workloads as W

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    wl = W.DISTANCE_WORKLOADS[args.workload]()
    spec = wl.scene
    scene = B.Scene()
    for kind in spec.order:
        getattr(scene, "add_" + kind)(*getattr(spec, kind).values())
    scene.commit()
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    per_query = 24 + 8  # point in, distance out
    if args.workload == "distance_queries":
        qs = {}
        for k, (ids, pts) in wl.meta["queries"].items():
            if rank > 0:  # weak scaling: each rank its own rotation of the queries
                sh = (rank * 7919) % len(ids)
                ids, pts = np.roll(ids, sh), np.roll(pts, sh, 0)
            qs[k] = (torch.from_numpy(ids.astype(np.int32)).to(dev), torch.from_numpy(pts).to(dev))
        n = sum(int(i.shape[0]) for i, _ in qs.values())
        outs = {k: torch.empty(i.shape[0], dtype=torch.float64, device=dev)
                for k, (i, _) in qs.items()}
        lib = scene._lib

        def launch(k, ev=None):
            ids, pts = qs[k]
            B._check(lib.bzr_distance_to_surface(scene._h, B.KIND_NAMES.index(k), ids.shape[0],
                                                 ids.data_ptr(), pts.data_ptr(),
                                                 outs[k].data_ptr(), None,
                                                 B.C.c_void_p(stream.cuda_stream)))

        kinds = list(qs)
        launches = len(kinds)
        alg = {k: int(qs[k][0].shape[0]) * (4 + 4 + per_query + DIST_RECORD_BYTES[k]) for k in kinds}
    else:
        pts_np = wl.meta["points"]
        if rank > 0:
            pts_np = np.roll(pts_np, (rank * 7919) % len(pts_np), 0)
        pts = torch.from_numpy(pts_np).to(dev)
        n = int(pts.shape[0])
        out = dict(distance=torch.empty(n, dtype=torch.float64, device=dev),
                   prim=torch.empty(n, dtype=torch.int32, device=dev),
                   geom=torch.empty(n, dtype=torch.int32, device=dev))
        lib = scene._lib

        def launch(k, ev=None):
            B._check(lib.bzr_closest_surface(scene._h, n, pts.data_ptr(),
                                             out["distance"].data_ptr(), out["prim"].data_ptr(),
                                             out["geom"].data_ptr(),
                                             B.C.c_void_p(stream.cuda_stream)))

        kinds = ["scene"]
        launches = 1
        alg = {"scene": n * (per_query + 8)}

    def step(evs=None):
        for j, k in enumerate(kinds):
            if evs is not None:
                evs[j].record(stream)
            launch(k)
        if evs is not None:
            evs[-1].record(stream)

    for i in range(args.warmup):
        flush.fill_(i & 0xFF)
        step()
    torch.cuda.synchronize(dev)
    scene.check()
    if pg:
        pg.barrier()
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(len(kinds) + 1)]
           for _ in range(args.steps)]
    for i in range(args.steps):
        flush.fill_((i + 1) & 0xFF)
        step(evs[i])
    torch.cuda.synchronize(dev)
    clocks = sampler.stop() if sampler else None
    scene.check()
    per_kind_ms = {k: sum(e[j].elapsed_time(e[j + 1]) for e in evs) / args.steps
                   for j, k in enumerate(kinds)}
    total_ms = sum(per_kind_ms.values()) * args.steps
    if pg:
        total_ms = multi.max_over_ranks(total_ms)
    value = world * n * args.steps / (total_ms / 1e3) / 1e6
    top = max(per_kind_ms, key=per_kind_ms.get)
    achieved = alg[top] / (per_kind_ms[top] / 1e3) / 1e9
    peak, peak_src = load_peaks()

    e2e = None
    if not args.no_e2e:
        if args.workload == "distance_queries":
            host = {k: (torch.from_numpy(ids.cpu().numpy().view(np.uint32)).pin_memory(),
                        torch.from_numpy(p.cpu().numpy()).pin_memory()) for k, (ids, p) in qs.items()}
            hout = {k: torch.empty(i.shape[0], dtype=torch.float64).pin_memory() for k, (i, _) in host.items()}

            def e2e_step():
                for k, (ids, p) in host.items():
                    B._check(lib.bzr_distance_to_surface(
                        scene._h, B.KIND_NAMES.index(k), ids.shape[0], ids.data_ptr(),
                        p.data_ptr(), hout[k].data_ptr(), None, None))
            h2d, d2h = n * 28, n * 8
        else:
            hp = torch.from_numpy(pts.cpu().numpy()).pin_memory()
            hd = torch.empty(n, dtype=torch.float64).pin_memory()
            hpr = torch.empty(n, dtype=torch.int32).pin_memory()
            hg = torch.empty(n, dtype=torch.int32).pin_memory()

            def e2e_step():
                B._check(lib.bzr_closest_surface(scene._h, n, hp.data_ptr(), hd.data_ptr(),
                                                 hpr.data_ptr(), hg.data_ptr(), None))
            h2d, d2h = n * 24, n * 16
        for _ in range(max(1, args.warmup)):
            e2e_step()
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        el = time.perf_counter() - t0
        if pg:
            el = multi.max_over_ranks(el)
        e2e = {"value": world * n * args.steps / el / 1e6, "unit": "Mqueries/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.workload, args.cpu_seconds)
        if "value" in cpu:
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if rank == 0:
        cfg = {"workload": args.workload, "queries_per_gpu": n,
               "scene": {k: len(next(iter(getattr(spec, k).values()))) for k in spec.order},
               "parallelism": f"replicated-scene x{world}",
               "l2": "flushed between timed steps (256 MiB write)"}
        print(json.dumps({
            "metric": ("Mqueries/s distance_to_surface (per-primitive, bit-exact) on 1 B200"
                       if args.workload == "distance_queries" else
                       "Mqueries/s nearest surface over the scene (bit-exact) on 1 B200"),
            "value": value, "unit": "Mqueries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": cfg,
            "ms_per_kind": per_kind_ms, "e2e": e2e, "gpu_launches": args.steps * launches,
            "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "peak_source": peak_src},
            "cpu_baseline": cpu, "clocks": clocks}), flush=True)
    if pg:
        pg.destroy_process_group()
    return 0


def main(argv=None):
    args = parse(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload in ("batched_icospheres", "adjoint_scene") and args.mode == "both":
        args.mode = "fp64"  # these forms time one path per run
    if args.workload == "batched_icospheres":
        return run_batched(args)
    if args.workload == "adjoint_scene":
        return run_adjoint(args)
    if args.workload in ("distance_queries", "closest_surface"):
        return run_distance(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
