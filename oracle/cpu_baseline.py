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
                seconds_per_batch=med, rays=rays.n, repetitions=len(times))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="mixed_primitives")
    ap.add_argument("--seconds", type=float, default=10.0)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--max-rays", type=int, default=0)
    ap.add_argument("--min-reps", type=int, default=3)
    a = ap.parse_args(argv)
    print(json.dumps(measure(a.workload, a.seconds, a.threads, a.max_rays, a.min_reps)))


if __name__ == "__main__":
    main()
