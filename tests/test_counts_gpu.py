"""The kernels' work counters on the GPU (bzr_work_counts_ex) equal the CPU emulator's, which
runs the same per-ray code compiled for the host: every box-test decision, node fetch, leaf
fetch and primitive test of the FP64 and the mixed walk is the same on both, so the FP32 test
of the wide nodes decodes the quantised boxes on the device exactly as on the host."""
import numpy as np
import pytest

from blazert_b200 import workloads as W
from tests.emu.emu import EmuScene
from tests.helpers import product_scene, uncovered_workload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["icosphere_pinhole", "mixed_primitives", "heightfield",
                                  "uncovered_rays"])
def test_device_counts_equal_emulator(name, mode):
    """(uncovered_rays: rays the mixed passes hand to their FP64 passes, which count them.)"""
    import torch

    kw = {"n_rays": 200_000}
    if name == "heightfield":
        kw["grid"] = 512
    if name == "icosphere_pinhole":
        kw = {}
    if name == "uncovered_rays":
        wl = uncovered_workload()[0]
    else:
        wl = W.WORKLOADS[name](**kw)
    R = wl.rays
    s = product_scene(wl.scene)
    dev = torch.device("cuda", 0)
    o, d = torch.from_numpy(R.origins).to(dev), torch.from_numpy(R.directions).to(dev)
    tmn, tmx = torch.from_numpy(R.tmin).to(dev), torch.from_numpy(R.tmax).to(dev)
    got = s.work_counts(o, d, tmn, tmx, mode=mode)
    want = EmuScene(wl.scene).work_counts(R.origins, R.directions, R.tmin, R.tmax, mode=mode)
    assert got == want
    s.close()
