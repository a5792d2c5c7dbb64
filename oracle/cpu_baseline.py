"""Times the reference's own intersect1 loop on the host CPU (TEST/BASELINE INFRASTRUCTURE).

    python -m oracle.cpu_baseline --workload mixed_primitives --seconds 10 [--threads N]

Uses oracle/_ref/libref_bench.so (the reference headers compiled with its release flags and
OpenMP, rows of 512 rays with schedule(dynamic, 1) as examples/scene_primitives/main.cc:86-88
does) when it exists ("kind": "reference"), otherwise the C restatement ("kind": "port").
Prints one JSON object.  Run as a separate process so that its OpenMP runtime is not shared
with a CUDA process.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from blazert_b200 import workloads as W  # noqa: E402
from oracle.oracle import Oracle, RefScene  # noqa: E402


def host_cpu():
    """CPU model (from /proc/cpuinfo where it exists) and the count of logical CPUs."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


def measure(workload="mixed_primitives", seconds=10.0, threads=0, max_rays=0, min_reps=3,
            flavour="bench"):
    wl = W.WORKLOADS[workload]()
    rays = wl.rays if not max_rays else wl.rays.slice(0, max_rays)
    threads = threads or os.cpu_count() or 1
    kind = "reference" if RefScene.available(flavour) else "port"
    if kind == "reference":
        sc = RefScene(wl.scene, flavour=flavour)
        run = lambda: sc.intersect(rays.origins, rays.directions, rays.tmin, rays.tmax,
                                   nthreads=threads)["seconds"]
    else:
        sc = Oracle(wl.scene)

        def run():
            t0 = time.perf_counter()
            sc.intersect(rays.origins, rays.directions, rays.tmin, rays.tmax, nthreads=threads)
            return time.perf_counter() - t0
    run()  # warm-up
    times = []
    t_end = time.perf_counter() + seconds
    while len(times) < min_reps or time.perf_counter() < t_end:
        times.append(run())
        if len(times) >= 1000:
            break
    med = statistics.median(times)
    return dict(value=rays.n / med / 1e6, unit="Mrays/s", cores=threads, kind=kind,
                sample=f"{workload}: {rays.n} rays x {len(times)} repetitions "
                       f"({sum(times):.1f} s of CPU ray loop), median",
                seconds_per_batch=med, rays=rays.n, repetitions=len(times), **host_cpu())


def measure_distance(workload="distance_queries", seconds=10.0, threads=0, max_queries=0,
                     min_reps=3, flavour="bench"):
    """The reference's distance_to_surface over the per-primitive queries of each kind
    (distance_queries), or the nearest surface by a loop over every primitive with the
    reference's distance functions (closest_surface; the reference has no scene-level query),
    OpenMP over the queries.  Queries per second over the sample."""
    import ctypes as C

    import numpy as np

    from oracle.oracle import _dp, _ptr, _u32p

    wl = W.DISTANCE_WORKLOADS[workload]()
    threads = threads or os.cpu_count() or 1
    sc = RefScene(wl.scene, flavour=flavour)
    lib = sc._lib
    lib.ref_distance_to_surface_timed.restype = C.c_double
    lib.ref_distance_to_surface_timed.argtypes = [C.c_void_p, C.c_int, C.c_long, _u32p, _dp,
                                                  _dp, C.c_int]
    lib.ref_closest_surface_timed.restype = C.c_double
    lib.ref_closest_surface_timed.argtypes = [C.c_void_p, C.c_long, _dp, _dp, _u32p, _u32p,
                                              C.c_int]
    kinds = ("mesh", "spheres", "planes", "cylinders")
    if workload == "distance_queries":
        qs = {k: (ids[:max_queries or None], np.ascontiguousarray(pts[:max_queries or None]))
              for k, (ids, pts) in wl.meta["queries"].items()}
        n = sum(len(i) for i, _ in qs.values())
        outs = {k: np.empty(len(i)) for k, (i, _) in qs.items()}

        def run():
            return sum(lib.ref_distance_to_surface_timed(
                sc._h, kinds.index(k), len(ids), _ptr(np.ascontiguousarray(ids, np.uint32), _u32p),
                _ptr(pts, _dp), _ptr(outs[k], _dp), threads) for k, (ids, pts) in qs.items())
        what = f"{workload}: {n} (primitive, point) pairs over {len(qs)} kinds"
    else:
        pts = np.ascontiguousarray(wl.meta["points"][:max_queries or 2048])
        n = len(pts)
        d, p_, g = np.empty(n), np.empty(n, np.uint32), np.empty(n, np.uint32)

        def run():
            return lib.ref_closest_surface_timed(sc._h, n, _ptr(pts, _dp), _ptr(d, _dp),
                                                 _ptr(p_, _u32p), _ptr(g, _u32p), threads)
        what = (f"{workload}: {n} points, each against every primitive with the reference's "
                "distance functions")
    run()
    times = []
    t_end = time.perf_counter() + seconds
    while len(times) < min_reps or time.perf_counter() < t_end:
        times.append(run())
        if len(times) >= 1000:
            break
    med = statistics.median(times)
    return dict(value=n / med / 1e6, unit="Mqueries/s", cores=threads, kind="reference",
                sample=f"{what} x {len(times)} repetitions ({sum(times):.1f} s), median",
                seconds_per_batch=med, queries=n, repetitions=len(times))


def measure_batched(seconds=10.0, threads=0, max_rays=0, min_reps=3, flavour="bench", stride=8):
    """The batching workload's sample: every `stride`-th of its 256 scenes (the level mix of the
    whole batch) with its own rays (at most max_rays per scene when given), each scene's
    intersect1 loop in turn; Mrays/s over the sample's rays.  The scenes' BVH builds are not
    timed."""
    wls = W.batched_icospheres()[::stride]
    threads = threads or os.cpu_count() or 1
    kind = "reference" if RefScene.available(flavour) else "port"
    runs = []
    for w in wls:
        rays = w.rays if not max_rays else w.rays.slice(0, min(max_rays, w.rays.n))
        if kind == "reference":
            sc = RefScene(w.scene, flavour=flavour)
            runs.append((rays, lambda sc=sc, r=rays: sc.intersect(
                r.origins, r.directions, r.tmin, r.tmax, nthreads=threads)["seconds"]))
        else:
            sc = Oracle(w.scene)

            def run(sc=sc, r=rays):
                t0 = time.perf_counter()
                sc.intersect(r.origins, r.directions, r.tmin, r.tmax, nthreads=threads)
                return time.perf_counter() - t0
            runs.append((rays, run))
    n = sum(r.n for r, _ in runs)
    for _, run in runs:  # warm-up
        run()
    times = []
    t_end = time.perf_counter() + seconds
    while len(times) < min_reps or time.perf_counter() < t_end:
        times.append(sum(run() for _, run in runs))
        if len(times) >= 1000:
            break
    med = statistics.median(times)
    return dict(value=n / med / 1e6, unit="Mrays/s", cores=threads, kind=kind,
                sample=f"batched_icospheres: every {stride}th scene ({len(runs)} scenes, "
                       f"{n} rays) x {len(times)} repetitions ({sum(times):.1f} s of CPU ray "
                       f"loop), median",
                seconds_per_batch=med, rays=n, repetitions=len(times), **host_cpu())


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="mixed_primitives")
    ap.add_argument("--seconds", type=float, default=10.0)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--max-rays", type=int, default=0)
    ap.add_argument("--min-reps", type=int, default=3)
    a = ap.parse_args(argv)
    if a.workload == "batched_icospheres":
        print(json.dumps(measure_batched(a.seconds, a.threads, a.max_rays, a.min_reps)))
    elif a.workload in W.DISTANCE_WORKLOADS:
        print(json.dumps(measure_distance(a.workload, a.seconds, a.threads, a.max_rays,
                                          a.min_reps)))
    else:
        print(json.dumps(measure(a.workload, a.seconds, a.threads, a.max_rays, a.min_reps)))


if __name__ == "__main__":
    main()
