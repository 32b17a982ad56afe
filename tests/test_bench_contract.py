"""bench.py's reference arm on CPU: the JSON line the driver reads (its keys and units, the
reference's own solver timed on the host cores), and that under torchrun only rank 0 runs it.
A small grid keeps it to about a second; the GPU arm runs in the GPU tiers."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

BENCH = os.path.join(ROOT, "bench.py")


def run(extra_env=None, *args):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, BENCH, "--impl", "reference", "--size", "24", "--steps", "2",
                           "--warmup", "1", *args], capture_output=True, text=True, env=env, timeout=300)


@pytest.mark.timeout(300)
def test_reference_arm_json_line():
    p = run()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    metric = "BiCGSTAB solves/sec to 1e-8 rel. residual + HBM GB/s; mixed/batched vs FP64"
    assert d["impl"] == "reference" and d["metric"] == metric
    assert d["unit"] == "solves/s" and d["higher_is_better"] is True and d["value"] > 0
    for k in ("n_gpus", "steps", "warmup", "ms_per_step", "scaling", "vs_baseline", "dtype", "data", "config"):
        assert k in d, k
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"] and cb["kind"] in ("reference", "port")
    assert cb["cores"] >= 1 and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


@pytest.mark.timeout(120)
def test_reference_arm_other_ranks_exit_quietly():
    p = run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0
    assert not [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
