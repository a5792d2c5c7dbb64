"""The batching form (bzr_batch_*): many scenes of uneven sizes in one launch per kind,
replayed from a CUDA graph; every scene's results equal the oracle's for that scene."""
import numpy as np
import pytest

import blazert_b200 as B
from blazert_b200 import workloads as W
from oracle.oracle import Oracle
from tests.helpers import mismatches, product_scene, to_numpy

pytestmark = pytest.mark.gpu


def _batch_case(n_scenes=24, scale=0.02, seed=4):
    wls = W.batched_icospheres(n_scenes=n_scenes, seed=seed, scale=scale)
    extra = W.mixed_primitives(n_rays=3000, n_spheres=500, n_cylinders=50, n_planes=20, seed=9)
    wls.insert(3, extra)                                  # a scene with three kinds
    wls.insert(5, W.Workload("empty", W.SceneSpec().add_spheres(np.zeros((0, 3)), np.zeros(0)),
                             W.RayBatch(np.zeros((50, 3)), np.ones((50, 3)))))  # nothing to hit
    wls.insert(7, W.Workload("no_rays", wls[0].scene, W.RayBatch(np.zeros((0, 3)), np.zeros((0, 3)))))
    return wls


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_batch_matches_per_scene_oracle(mode):
    import torch

    wls = _batch_case()
    scenes = [product_scene(w.scene) for w in wls]
    batch = B.Batch(scenes)
    offs = np.concatenate([[0], np.cumsum([w.rays.n for w in wls])])
    o = torch.from_numpy(np.concatenate([w.rays.origins for w in wls])).cuda()
    d = torch.from_numpy(np.concatenate([w.rays.directions for w in wls])).cuda()
    ts = torch.zeros(len(wls) + 1, dtype=torch.int64, device="cuda")
    for _ in range(3):  # first call captures the graph, later calls replay it
        out = batch.intersect(offs, o, d, timestamps=ts, mode=mode)
        assert batch.check() == 0
        got = to_numpy(out)
        for s, w in enumerate(wls):
            a, b = offs[s], offs[s + 1]
            ref = Oracle(w.scene).intersect(w.rays.origins, w.rays.directions)
            assert mismatches({k: v[a:b] for k, v in got.items()}, ref) == [], (s, w.name)
    t = ts.cpu().numpy()
    start = t[-1]
    for s, w in enumerate(wls):
        if w.rays.n and any(len(next(iter(getattr(w.scene, k).values()))) for k in w.scene.order):
            assert t[s] >= start > 0


def test_batch_tuning_changes_speed_not_results():
    """The batch kernels' launch shape (threads per block, stack storage, stack depth, sort and
    the mixed mode's node width; bzr_batch_tune) and the batch autotuner's choice, in both
    modes, re-capture the graph and give the oracle's results."""
    import torch

    from blazert_b200.autotune import autotune_batch

    wls = _batch_case(n_scenes=10)
    scenes = [product_scene(w.scene) for w in wls]
    batch = B.Batch(scenes)
    offs = np.concatenate([[0], np.cumsum([w.rays.n for w in wls])])
    o = torch.from_numpy(np.concatenate([w.rays.origins for w in wls])).cuda()
    d = torch.from_numpy(np.concatenate([w.rays.directions for w in wls])).cuda()
    refs = [Oracle(w.scene).intersect(w.rays.origins, w.rays.directions) for w in wls]

    def check(mode="fp64"):
        got = to_numpy(batch.intersect(offs, o, d, mode=mode))
        assert batch.check() == 0
        for s, ref in enumerate(refs):
            a, b = offs[s], offs[s + 1]
            assert mismatches({k: v[a:b] for k, v in got.items()}, ref) == [], (s, mode)

    for cfg in (dict(threads=64), dict(threads=256), dict(shared_stack=True),
                dict(threads=128, shared_stack=False), dict(stack_depth=32), dict(sort=True),
                dict(sort=True, threads=64, stack_depth=64), dict(sort=False),
                dict(node_width=2), dict(node_width=2, sort=True), dict(node_width=8)):
        try:
            batch.tune(**cfg)
        except B.BlazertError as e:  # 32 entries only when every scene's tree fits them
            assert cfg == dict(stack_depth=32) and e.code == B.EINVAL
            assert "more than 32" in str(e)
            continue
        check()
        check("mixed")
    with pytest.raises(B.BlazertError) as e:
        batch.tune(node_width=4)
    assert e.value.code == B.EINVAL
    res = autotune_batch(batch, offs, o, d)
    assert set(res["choice"]) == {"threads", "shared_stack", "stack_depth", "sort"}
    check()
    res = autotune_batch(batch, offs, o, d, mode="mixed")
    assert set(res["choice"]) == {"threads", "shared_stack", "stack_depth", "sort", "node_width"}
    check("mixed")


def test_batch_full_size_matches_oracle():
    """The batching workload at its full size: 256 perturbed icospheres (levels 3-7), each with
    its own log-uniform ray batch (about 36M rays in all), in one graph replay per mode; every
    scene's results equal the oracle's (OpenMP over the host cores) bit for bit, in both modes
    and with the per-scene coherence sort on."""
    import torch

    wls = W.batched_icospheres()
    assert len(wls) == 256
    scenes = [product_scene(w.scene) for w in wls]
    batch = B.Batch(scenes)
    offs = np.concatenate([[0], np.cumsum([w.rays.n for w in wls])])
    assert offs[-1] > 30_000_000
    o = torch.from_numpy(np.concatenate([w.rays.origins for w in wls])).cuda()
    d = torch.from_numpy(np.concatenate([w.rays.directions for w in wls])).cuda()
    outs = {}
    for mode, sort in (("fp64", False), ("mixed", False), ("mixed", True)):
        batch.tune(sort=sort)
        outs[(mode, sort)] = to_numpy(batch.intersect(offs, o, d, mode=mode))
        assert batch.check() == 0
    for s, w in enumerate(wls):
        ref = Oracle(w.scene).intersect(w.rays.origins, w.rays.directions)
        a, b = offs[s], offs[s + 1]
        for key, got in outs.items():
            assert mismatches({k: v[a:b] for k, v in got.items()}, ref) == [], (s, key)
