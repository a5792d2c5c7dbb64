"""bench.py's reference arm on the CPU: `--impl reference` times the reference's own code (its
headers built against the blaze shim, oracle/_ref) on the host and prints one JSON line with the
contract's keys; under several ranks only rank 0 prints."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HAVE_REF = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_bench.so"))

KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "impl",
        "cpu_baseline", "e2e"}


def _run(args, env=None):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                       capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, **(env or {})))
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")]


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("workload", ["mixed_primitives", "distance_queries"])
def test_reference_arm_prints_the_contract_line(workload):
    lines = _run(["--impl", "reference", "--workload", workload, "--steps", "1", "--warmup", "1"])
    assert len(lines) == 1
    line = lines[0]
    assert KEYS <= set(line), KEYS - set(line)
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
def test_reference_arm_prints_nothing_on_other_ranks():
    assert _run(["--impl", "reference", "--steps", "1", "--warmup", "1"],
                env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []
