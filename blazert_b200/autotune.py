"""Picks a scene's speed knobs by timing them on a sample of the caller's rays.

The knobs (bzr_scene_tune) never change results, only the processing order and launch
shape, so tuning is safe to run on live data.  Each candidate is timed with CUDA events on
the caller's stream over `reps` repetitions after one warm-up; the fastest is kept.
"""
from __future__ import annotations

import itertools


def autotune(scene, origins, directions, tmin=None, tmax=None, mode="fp64", reps=3,
             sample=1 << 20, stream=None):
    """origins/directions: torch CUDA tensors (n x 3 float64).  Returns the chosen settings
    and the per-candidate timings (ms)."""
    import torch

    n = origins.shape[0]
    m = min(n, sample)
    o, d = origins[:m], directions[:m]
    tmn = None if tmin is None else tmin[:m]
    tmx = None if tmax is None else tmax[:m]
    st = stream or torch.cuda.current_stream(origins.device)
    candidates = [dict(sort=s) for s in (True, False)]
    timings = []
    out = None
    for cand in candidates:
        scene.tune(sort=cand["sort"], sort_min_rays=0 if cand["sort"] else None)
        out = scene.intersectN(o, d, tmn, tmx, mode=mode, out=out, stream=st)  # warm-up
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(reps)]
        for a, b in evs:
            a.record(st)
            scene.intersectN(o, d, tmn, tmx, mode=mode, out=out, stream=st)
            b.record(st)
        torch.cuda.synchronize(origins.device)
        timings.append(min(a.elapsed_time(b) for a, b in evs))
    best = min(range(len(candidates)), key=lambda i: timings[i])
    choice = candidates[best]
    scene.tune(sort=choice["sort"], sort_min_rays=1 << 16)
    return dict(choice=choice, timings_ms={str(c): t for c, t in zip(candidates, timings)},
                sample_rays=m)
