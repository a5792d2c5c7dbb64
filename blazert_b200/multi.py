"""Multi-GPU form: one process per GPU (launched by torchrun), the committed scene replicated on
every rank, rays split across ranks.  Rays are independent and the scene is read-only, so the
query itself needs no collective; the only exchanges are the optional all-gather of the hit
records (for callers that want every result on every rank) and the max-over-ranks of timings.

    ray_shard(n, rank, world)          contiguous, balanced [begin, end) of n rays for a rank
    rank_batch(origins, ..., rank)     per-rank batch of a weak-scaling run (fixed size per GPU)
    max_over_ranks(x, group)           all-reduce MAX of a host float (timings)
    intersect_sharded(trace, ...)      trace this rank's shard, all-gather the records

`trace` is any callable with the signature of Scene.intersectN on host arrays; the processes
use the backend of the default process group (NCCL on GPUs).
"""
from __future__ import annotations

import numpy as np

RESULT_KEYS = ("t", "uv", "normal", "prim", "geom", "hit")


def ray_shard(n: int, rank: int, world: int) -> tuple[int, int]:
    """Rays [begin, end) of `rank`: the first n % world ranks take one ray more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    q, r = divmod(n, world)
    begin = rank * q + min(rank, r)
    return begin, begin + q + (1 if rank < r else 0)


def rank_batch(origins, directions, tmin, tmax, rank: int):
    """Batch of `rank` in a weak-scaling run: every rank traces a batch of the full size, rank r
    the batch rotated by r * 7919 rays, so the ranks' batches differ but have the same
    statistics.  Rank 0 gets the batch unchanged."""
    n = origins.shape[0]
    sh = (rank * 7919) % n if n else 0
    if sh == 0:
        return origins, directions, tmin, tmax
    roll = lambda a: None if a is None else np.roll(a, sh, 0)  # noqa: E731
    return roll(origins), roll(directions), roll(tmin), roll(tmax)


def max_over_ranks(x: float, group=None) -> float:
    """MAX of x over the ranks of `group` (the default group when None; x itself when
    torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def intersect_sharded(trace, origins, directions, tmin=None, tmax=None, rank=0, world=1,
                      group=None, gather=True):
    """Traces rays ray_shard(n, rank, world) with `trace` and, when `gather`, all-gathers the
    records so that every rank returns the results of all n rays in input order (equal to a
    single trace of the whole batch).  Without `gather` each rank returns its own shard's
    records and its (begin, end)."""
    n = origins.shape[0]
    b, e = ray_shard(n, rank, world)
    part = trace(origins[b:e], directions[b:e], None if tmin is None else tmin[b:e],
                 None if tmax is None else tmax[b:e])
    part = {k: np.asarray(part[k]) for k in RESULT_KEYS}
    if not gather or world == 1:
        return part, (b, e)
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    full = {}
    for k in RESULT_KEYS:
        a = part[k]
        # shards differ in length by at most one ray: pad to the largest, gather, trim
        rows = -(-n // world)
        pad = np.zeros((rows,) + a.shape[1:], a.dtype)
        pad[: a.shape[0]] = a
        src = torch.from_numpy(pad.view(np.uint8)).to(dev)
        bufs = [torch.empty_like(src) for _ in range(world)]
        dist.all_gather(bufs, src, group=group)
        pieces = []
        for r in range(world):
            rb, re_ = ray_shard(n, r, world)
            got = bufs[r].cpu().numpy().view(a.dtype).reshape((rows,) + a.shape[1:])
            pieces.append(got[: re_ - rb])
        full[k] = np.concatenate(pieces, 0)
    return full, (0, n)
