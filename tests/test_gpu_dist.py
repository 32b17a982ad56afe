"""Row-partitioned solve of one system (fiim_dist_*) on B200.

* The emulation runs R row blocks in one process on one GPU through the per-rank kernels,
  with device copies in place of NCCL; at R = 1 it is the single-GPU solve bit for bit (the
  same products and the same reduction trees). At R > 1 only the dot products' summation
  order differs from one GPU, so the iteration count stays within +-2 of the single-GPU
  solve (the oracle's acceptance band), the termination code is the same and the solutions
  agree to the tolerance.
* The NCCL path itself is run at world size 1 (one GPU per process here): it must give the
  emulation's bits, with host and with device arrays.
"""
import numpy as np
import pytest
import torch

import fiim_b200 as FB
from conftest import load_golden

pytestmark = pytest.mark.gpu


def system(N=16, pe=0.5):
    A = FB.gen_convdiff3d(N, pe)
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, gpu=True)
    b = FB.rand_normal(len(A[0]) - 1, 20261203)
    return A, F, b


def single(A, F, b, variant="pdfiim", tol=1e-8, nmax=1000):
    x = np.zeros(len(b))
    S = FB.Solver(A, F, variant=variant)
    r = S.solve(b, x, tol=tol, nmax=nmax)
    S.close()
    return x, r


def emulate(A, F, b, world, variant="pdfiim", tol=1e-8, nmax=1000, row_starts=None):
    x = np.zeros(len(b))
    r = FB.dist_emulate(A, F, b, x, world, tol=tol, nmax=nmax, variant=variant, row_starts=row_starts)
    return x, r


def test_world1_is_the_single_gpu_solve(monkeypatch):
    monkeypatch.setenv("FIIM_PERSIST", "0")   # the launched-kernel path the emulation shares
    A, F, b = system(16)
    x1, r1 = single(A, F, b)
    xe, re = emulate(A, F, b, 1)
    assert np.array_equal(x1, xe)
    assert (r1["iter"], r1["info"], r1["resval"]) == (re["iter"], re["info"], re["resval"])


@pytest.mark.parametrize("world", [2, 3, 4, 7])
def test_row_blocks_agree_with_one_gpu(world):
    A, F, b = system(16)
    x1, r1 = single(A, F, b)
    xw, rw = emulate(A, F, b, world)
    dx = np.linalg.norm(xw - x1) / np.linalg.norm(x1)
    print(f"world {world}: iter {rw['iter']} (1 GPU {r1['iter']}), info {rw['info']}, "
          f"true relres {rw['true_relres']:.2e}, x diff {dx:.1e}")
    assert rw["info"] == r1["info"] == 0
    assert abs(rw["iter"] - r1["iter"]) <= 2
    assert rw["true_relres"] < 1e-7
    assert dx < 1e-6


@pytest.mark.parametrize("variant", ["afiim", "acifim"])
def test_variants_keep_their_control_constants(variant):
    A, F, b = system(12, 0.9)
    x1, r1 = single(A, F, b, variant=variant)
    xw, rw = emulate(A, F, b, 3, variant=variant)
    assert rw["info"] == r1["info"] and abs(rw["iter"] - r1["iter"]) <= 2
    assert np.linalg.norm(xw - x1) / np.linalg.norm(x1) < 1e-6


def test_nmax_stops_every_block_together():
    A, F, b = system(16)
    x1, r1 = single(A, F, b, nmax=7)
    xw, rw = emulate(A, F, b, 4, nmax=7)
    assert r1["info"] == rw["info"] == 3 and r1["iter"] == rw["iter"] == 7


def test_uneven_blocks_and_single_rows():
    """Blocks of one row at both ends and a large one between."""
    A, F, b = system(10)
    n = len(b)
    x1, r1 = single(A, F, b)
    for rs in ([0, 1, n - 1, n], [0, 1, 2, 3, n], [0, n // 3, n // 3 + 1, n]):
        xw, rw = emulate(A, F, b, len(rs) - 1, row_starts=np.array(rs))
        assert rw["info"] == 0 and abs(rw["iter"] - r1["iter"]) <= 2
        assert np.linalg.norm(xw - x1) / np.linalg.norm(x1) < 1e-6


def test_random_columns_all_ranks_exchange():
    """A Zipf matrix with random columns: every block's halo reaches every other block."""
    n = 20000
    A = FB.gen_zipf(n, FB.zipf_scale(n, sample=n, seed=21), seed=21)
    F = FB.pdfiim_build(A, 0.1, 1, 1, 1, 32, "I", "B", gpu=True)
    b = FB.rand_normal(n, 4)
    x1, r1 = single(A, F, b, variant="afiim")
    for world in (3, 5):
        xw, rw = emulate(A, F, b, world, variant="afiim")
        print(f"zipf world {world}: iter {rw['iter']} (1 GPU {r1['iter']}), info {rw['info']}")
        assert rw["info"] == r1["info"] == 0 and abs(rw["iter"] - r1["iter"]) <= 2
        assert np.linalg.norm(xw - x1) / np.linalg.norm(x1) < 1e-6


def test_sherman2_within_the_reference_envelope():
    """sherman2 with the reference's own PDFIIM factors (golden): each partition's iteration
    count lies within +-2 of the oracle's rounding envelope and ends with the oracle's info."""
    g = load_golden("sherman2")
    A = (g["Ai"], g["Aj"], g["Av"])
    F = {k: g["pdfiim_" + k] for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    b = g["b"]
    lo, hi = (int(v) for v in g["pdfiim_iter_env"])
    infos = set(g["meta"]["results"]["pdfiim"]["infos"])   # over the oracle's summation orders
    for world in (1, 2, 3):
        x, r = emulate(A, F, b, world, tol=1e-8, nmax=1200)
        print(f"sherman2 world {world}: iter {r['iter']} info {r['info']} envelope [{lo},{hi}] infos {infos}")
        assert r["info"] in infos
        if r["info"] == 0:
            assert lo - 2 <= r["iter"] <= hi + 2


def test_nccl_world1_matches_the_emulation():
    A, F, b = system(16)
    n = len(b)
    xe, re = emulate(A, F, b, 1)
    rs = np.array([0, n], np.int64)
    Al, Fl = FB.dist_local(A, F, rs, 0)
    D = FB.DistSolver(0, 1, FB.dist_unique_id(), rs, Al, Fl, variant="pdfiim", device=0)
    x = np.zeros(n)
    r = D.solve(b, x, tol=1e-8, nmax=1000)
    assert np.array_equal(x, xe)
    assert (r["iter"], r["info"], r["resval"]) == (re["iter"], re["info"], re["resval"])
    x2 = np.zeros(n)
    r2 = D.solve(b, x2, tol=1e-8, nmax=1000)     # a second solve on the same handle
    assert np.array_equal(x2, xe) and r2["iter"] == r["iter"]
    D.close()
    # device arrays
    Dd = FB.DistSolver(0, 1, FB.dist_unique_id(), rs, Al, Fl, variant="pdfiim", memory="device", device=0)
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    rd = Dd.solve(bd, xd, tol=1e-8, nmax=1000)
    torch.cuda.synchronize()
    assert np.array_equal(xd.cpu().numpy(), xe) and rd["iter"] == re["iter"]
    Dd.close()


def test_set_up_errors():
    A, F, b = system(6)
    n = len(b)
    x = np.zeros(n)
    with pytest.raises(FB.FiimError, match="owns no rows"):
        FB.dist_emulate(A, F, b, x, 2, row_starts=np.array([0, 0, n]))
    with pytest.raises(FB.FiimError):
        FB.dist_emulate(A, F, b, x, 2, variant="acifim", row_starts=np.array([0, n, n + 1]))


def test_bench_system_two_blocks():
    """The 128^3 system (n = 2,097,152) in two row blocks."""
    import time
    A, F, b = system(128)
    x1, r1 = single(A, F, b, nmax=1200)
    t0 = time.perf_counter()
    x2, r2 = emulate(A, F, b, 2, nmax=1200)
    dt = time.perf_counter() - t0
    dx = np.linalg.norm(x2 - x1) / np.linalg.norm(x1)
    print(f"128^3: 1 GPU iter {r1['iter']} {r1['device_ms']:.1f} ms; 2 blocks iter {r2['iter']} "
          f"{r2['device_ms']:.1f} ms device ({dt:.1f} s with set-up), x diff {dx:.1e}")
    assert r2["info"] == r1["info"] == 0 and abs(r2["iter"] - r1["iter"]) <= 2
    assert dx < 1e-6
