"""The multi-GPU host logic (blazert_b200.multi) with two gloo ranks on the CPU: shards cover
the batch exactly once, the all-gathered records equal one trace of the whole batch, and the
timing reduction takes the maximum.  The per-shard tracer here is the oracle (the checker); on
GPUs it is Scene.intersectN."""
import os
import socket

import numpy as np
import pytest

from blazert_b200 import multi


def test_ray_shard_partitions():
    for n in (0, 1, 7, 1000, 1 << 20):
        for world in (1, 2, 3, 8):
            spans = [multi.ray_shard(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[r][1] == spans[r + 1][0] for r in range(world - 1))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        multi.ray_shard(10, 2, 2)


def test_rank_batch_rotates_except_rank0():
    o = np.arange(30.0).reshape(10, 3)
    d = o + 1
    assert multi.rank_batch(o, d, None, None, 0)[0] is o
    o1, d1, t0, t1 = multi.rank_batch(o, d, None, None, 1)
    assert t0 is None and t1 is None
    assert np.array_equal(o1, np.roll(o, 7919 % 10, 0)) and np.array_equal(d1, np.roll(d, 7919 % 10, 0))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from blazert_b200 import workloads as W
    from oracle.oracle import Oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wl = W.mixed_primitives(n_rays=5001, seed=12)
        R = wl.rays
        ora = Oracle(wl.scene)
        trace = lambda o, d, a, b: ora.intersect(o, d, a, b)  # noqa: E731
        full, span = multi.intersect_sharded(trace, R.origins, R.directions, R.tmin, R.tmax,
                                             rank=rank, world=world)
        own, own_span = multi.intersect_sharded(trace, R.origins, R.directions, R.tmin, R.tmax,
                                                rank=rank, world=world, gather=False)
        m = multi.max_over_ranks(1.5 + rank)
        if rank == 0:
            ref = ora.intersect(R.origins, R.directions, R.tmin, R.tmax)
            same = all(np.array_equal(full[k].view(np.uint8), np.asarray(ref[k]).view(np.uint8))
                       for k in multi.RESULT_KEYS)
            q.put((same, span, own_span, own["t"].shape[0], m))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_gather_and_max():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    same, span, own_span, own_n, m = q.get(timeout=10)
    assert same
    assert span == (0, 5001) and own_span == (0, 2501) and own_n == 2501
    assert m == 2.5
