"""Picks a scene's speed knobs by timing them on a sample of the caller's rays.

The knobs (bzr_scene_tune) never change results, only the processing order and the launch
shape, so tuning is safe to run on live data:

  sort          coherence sort of each batch (octant + origin Morton order) or caller order
  threads       threads per block of the traversal kernels: 64, 128, 256
  shared_stack  traversal stack in shared memory (sized from the tree) or thread-local
  chunk         rays a warp takes from the work counter per fetch: 32, 64, 128, or 0 for
                exactly the lanes that are idle
  top_nodes     top-level nodes each block stages in shared memory: 0, 64, 256

The search is coordinate-wise: starting from the defaults, each knob in turn is set to the
value with the lowest time while the others stay at their current best; two sweeps.  Each
candidate is timed with CUDA events on the caller's stream, the minimum over `reps`
repetitions after one warm-up.  The tree's node width stays binary: the reference's visit
order, and so its tie-breaking, is defined on its binary tree.
"""
from __future__ import annotations

KNOBS = {"sort": (False, True), "threads": (128, 64, 256), "shared_stack": (False, True),
         "chunk": (32, 0, 64, 128), "top_nodes": (0, 64, 256)}


def autotune(scene, origins, directions, tmin=None, tmax=None, mode="fp64", reps=3,
             sample=1 << 20, stream=None, knobs=None, sweeps=2):
    """origins/directions: torch CUDA tensors (n x 3 float64).  Applies and returns the chosen
    settings with the per-candidate timings (ms)."""
    import torch

    knobs = dict(KNOBS if knobs is None else knobs)
    n = origins.shape[0]
    m = min(n, sample)
    o, d = origins[:m], directions[:m]
    tmn = None if tmin is None else tmin[:m]
    tmx = None if tmax is None else tmax[:m]
    st = stream or torch.cuda.current_stream(origins.device)
    out = None
    timings = {}

    def apply(cfg):
        scene.tune(sort=cfg["sort"], sort_min_rays=0 if cfg["sort"] else 1 << 16,
                   threads=cfg["threads"], shared_stack=cfg["shared_stack"], chunk=cfg["chunk"],
                   top_nodes=cfg.get("top_nodes", 0))

    def timed(cfg):
        nonlocal out
        key = str(sorted(cfg.items()))
        if key in timings:
            return timings[key]
        try:
            apply(cfg)
        except Exception:  # e.g. the stack does not fit shared memory at this block size
            timings[key] = float("inf")
            return timings[key]
        out = scene.intersectN(o, d, tmn, tmx, mode=mode, out=out, stream=st)  # warm-up
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(reps)]
        for a, b in evs:
            a.record(st)
            scene.intersectN(o, d, tmn, tmx, mode=mode, out=out, stream=st)
            b.record(st)
        torch.cuda.synchronize(origins.device)
        timings[key] = min(a.elapsed_time(b) for a, b in evs)
        return timings[key]

    best = {k: v[0] for k, v in knobs.items()}
    for _ in range(sweeps):
        for k, values in knobs.items():
            scores = {v: timed({**best, k: v}) for v in values}
            best[k] = min(scores, key=scores.get)
    apply(best)
    return dict(choice=best, best_ms=timings[str(sorted(best.items()))],
                timings_ms=timings, sample_rays=m)


BATCH_KNOBS = {"threads": (128, 64, 256), "shared_stack": (False, True), "stack_depth": (64, 32),
               "sort": (False, True), "node_width": (8, 2)}


def autotune_batch(batch, ray_offsets, origins, directions, tmin=None, tmax=None, mode="fp64",
                   reps=3, stream=None, knobs=None):
    """The batching form's knobs (threads per block, stack storage, entries of the thread-local
    stack, per-scene coherence sort and, in the mixed mode, the node width of the walk), timed
    on the caller's whole batch (each candidate captures its own graph, then replays it `reps`
    times).  A candidate the batch refuses (a stack that does not fit) scores infinity.
    Applies and returns the choice with the per-candidate timings (ms)."""
    import torch

    knobs = dict(BATCH_KNOBS if knobs is None else knobs)
    if mode != "mixed":
        knobs.pop("node_width", None)  # the FP64 mode always walks the binary nodes
    st = stream or torch.cuda.current_stream(origins.device)
    out = None
    timings = {}

    def timed(cfg):
        nonlocal out
        key = str(sorted(cfg.items()))
        if key in timings:
            return timings[key]
        try:
            batch.tune(**cfg)
        except Exception:  # e.g. the stack does not fit shared memory at this block size
            timings[key] = float("inf")
            return timings[key]
        out = batch.intersect(ray_offsets, origins, directions, tmin, tmax, out=out, mode=mode,
                              stream=st)  # capture + warm-up
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(reps)]
        for a, b in evs:
            a.record(st)
            batch.intersect(ray_offsets, origins, directions, tmin, tmax, out=out, mode=mode,
                            stream=st)
            b.record(st)
        torch.cuda.synchronize(origins.device)
        timings[key] = min(a.elapsed_time(b) for a, b in evs)
        return timings[key]

    best = {k: v[0] for k, v in knobs.items()}
    for k, values in knobs.items():
        scores = {v: timed({**best, k: v}) for v in values}
        best[k] = min(scores, key=scores.get)
    batch.tune(**best)
    return dict(choice=best, best_ms=timings[str(sorted(best.items()))], timings_ms=timings)


HOST_KNOBS = {"host_min_chunk": (1 << 17, 1 << 16, 1 << 15, 1 << 14),
              "host_chunks": (8, 4, 6, 12, 16), "host_grid_div": (1, 2, 3),
              "host_edge": (0, 1 << 16, 1 << 17)}


def autotune_host(scene, origins, directions, tmin=None, tmax=None, out=None, mode="fp64",
                  reps=3, knobs=None, sweeps=2):
    """The pipeline of host-array calls (bzr_scene_tune HOST_MIN_CHUNK / HOST_CHUNKS /
    HOST_GRID_DIV / HOST_EDGE): the smallest chunk and how many chunks the batch is split into,
    what share of the grid each chunk's kernels take and the size of small first and last
    chunks, timed
    end to end (wall clock, host arrays, copies included) on the caller's whole batch.  The
    device-path knobs stay as they are.  Applies and returns the choice with the timings (ms)."""
    import time

    knobs = dict(HOST_KNOBS if knobs is None else knobs)
    timings = {}

    def timed(cfg):
        nonlocal out
        key = str(sorted(cfg.items()))
        if key in timings:
            return timings[key]
        scene.tune(**cfg)
        out = scene.intersectN(origins, directions, tmin, tmax, mode=mode, out=out)  # warm-up
        best = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            scene.intersectN(origins, directions, tmin, tmax, mode=mode, out=out)
            best = min(best, (time.perf_counter() - t0) * 1e3)
        timings[key] = best
        return best

    best = {k: v[0] for k, v in knobs.items()}
    for _ in range(sweeps):
        for k, values in knobs.items():
            scores = {v: timed({**best, k: v}) for v in values}
            best[k] = min(scores, key=scores.get)
    scene.tune(**best)
    return dict(choice=best, best_ms=timings[str(sorted(best.items()))], timings_ms=timings)
