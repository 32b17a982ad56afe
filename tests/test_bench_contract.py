"""bench.py on CPU: the reference arm's JSON line (its keys and units, the reference's own
solver timed on the host cores, no library of this project loaded), that under torchrun only
rank 0 runs it, that the numpy-built workload of that arm is the library's bit for bit, and
that `--gpus N` starts N ranks and reports the max over ranks (a gloo dry run). A small grid
keeps it to seconds; the GPU arm runs in the GPU tiers."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT
import fiim_b200 as FB

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
    sys.path.insert(0, ROOT)
    import bench
    assert d["config"] == bench.config(24, 7 * 24 ** 3 - 6 * 24 ** 2)   # the GPU arm's config, key for key
    # the process that timed the reference loaded no library of this project but the reference's
    assert not [p for p in d["libraries_loaded"] if "libfiim_b200" in p]
    if d["cpu_baseline"]["kind"] == "reference":
        assert os.path.join("oracle", "_ref", "libref_pdfiim.so") in d["libraries_loaded"]
        assert "full solves" in d["cpu_baseline"]["sample"] and d["iterations"] > 0
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


@pytest.mark.parametrize("N", [1, 2, 7, 24])
def test_reference_arm_workload_is_the_librarys(N):
    """The reference arm builds the system with numpy; it must be the GPU arm's bit for bit."""
    sys.path.insert(0, ROOT)
    import bench
    A, b = bench.workload_host(N)
    A2 = FB.gen_convdiff3d(N, 0.5)
    assert all(x.dtype == y.dtype and np.array_equal(x, y) for x, y in zip(A, A2))
    assert np.array_equal(b, FB.rand_normal(N ** 3, bench.SEED))
    big = bench.rand_normal_host(300000, 12345)
    assert np.array_equal(big, FB.rand_normal(300000, 12345))


@pytest.mark.timeout(300)
def test_gpus_flag_starts_the_ranks():
    """`bench.py --gpus 2` without torchrun starts 2 ranks; rank 0 prints the max over ranks
    (rank 1's steps take 20 ms, rank 0's 10 ms)."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    p = subprocess.run([sys.executable, BENCH, "--gpus", "2", "--steps", "5", "--warmup", "3", "--dry-run"],
                       capture_output=True, text=True, env=env, timeout=240)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["dry_run"] is True and d["n_gpus"] == 2 and d["steps"] == 5
    assert d["ms_per_step"] >= 19.0 and d["rank0_ms_per_step"] < d["ms_per_step"]
    assert "rank 1 of 2" in p.stderr


def test_gpus_flag_disagreeing_with_world_size_gives_no_result():
    env = dict(os.environ, WORLD_SIZE="3", RANK="0", LOCAL_RANK="0")
    p = subprocess.run([sys.executable, BENCH, "--gpus", "2", "--dry-run"], capture_output=True, text=True,
                       env=env, timeout=60)
    assert p.returncode == 2 and not [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
