"""Mixed precision on B200: an FP32 BiCGSTAB with FP64 residual replacement (reliable updates,
the default) or FP64 iterative refinement around it (reliable = 0), with the factors G, H
stored in FP32 or BF16 and D^-1 in FP32.

The outer residual is recomputed in FP64, so the tolerance reached is FP64-verified: the
test recomputes ||b - A x|| / ||b|| with scipy on the host. The relative error against the
oracle's FP64 solution of the same system is reported and bounded by what the system's
conditioning allows at the residual reached.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import fiim_b200 as FB
import pyoracle as O
from conftest import sub

pytestmark = pytest.mark.gpu


def relres(A, b, x):
    n = len(b)
    M = sp.csr_matrix((A[2], A[1], A[0]), shape=(n, n))
    return np.linalg.norm(b - M @ x) / np.linalg.norm(b)


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
@pytest.mark.parametrize("name,prefix,variant", [("convdiff16_pdfiim", "", "pdfiim"),
                                                 ("poisson128_afiim", "", "afiim"),
                                                 ("convdiff2d48_acifim", "", "acifim")])
def test_mixed_reaches_fp64_tolerance(golden, name, prefix, variant, precision):
    g = golden(name)
    A = (g["Ai"], g["Aj"], g["Av"])
    F = {k: v for k, v in sub(g, prefix).items() if k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    S = FB.Solver(A, F, variant=variant, precision=precision, inner_tol=1e-5, reliable=0.0)
    x = np.zeros(len(g["b"]))
    r = S.solve(g["b"], x, tol=1e-10, nmax=5000)
    tr = relres(A, g["b"], x)
    xo, *_ = O.bicgstab(variant, A, g["b"], F, tol=1e-12, nmax=5000)
    err = np.linalg.norm(x - xo) / np.linalg.norm(xo)
    print(f"{name} {precision}: steps {r['refine_steps']} inner its {r['iter']} info {r['info']} "
          f"true relres {tr:.2e} (reported {r['true_relres']:.2e}) err vs FP64 oracle {err:.2e}")
    assert r["info"] == 0
    assert tr <= 1e-10 and abs(tr - r["true_relres"]) <= 1e-3 * tr + 1e-16
    assert r["refine_steps"] >= 2
    assert err <= 1e-6
    S.close()


def test_mixed_matches_fp64_solution_at_scale():
    """64^3 convection-diffusion with the library's own PDFIIM factors: FP32 and BF16 mixed
    solves (the default form, reliable updates) to 1e-10 against the FP64 GPU solve to 1e-12."""
    A = FB.gen_convdiff3d(64, 0.5)
    b = FB.rand_normal(64 ** 3, 20261203)
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    S64 = FB.Solver(A, F, variant="pdfiim")
    x64 = np.zeros(len(b))
    r64 = S64.solve(b, x64, tol=1e-12, nmax=2000)
    assert r64["info"] == 0
    for precision in ("fp32", "bf16"):
        S = FB.Solver(A, F, variant="pdfiim", precision=precision)
        x = np.zeros(len(b))
        r = S.solve(b, x, tol=1e-10, nmax=5000)
        err = np.linalg.norm(x - x64) / np.linalg.norm(x64)
        print(f"64^3 {precision}: {r} err vs FP64 {err:.2e}; FP64 to 1e-12: {r64['iter']} its")
        assert r["info"] == 0 and relres(A, b, x) <= 1e-10 and err <= 1e-8
        S.close()
    S64.close()


def test_mixed_reports_failure_to_converge():
    """A refinement step that does not reduce the FP64 residual ends the solve (not a hang)."""
    A = FB.gen_poisson2d(16)
    n = 256
    I = np.arange(n + 1, dtype=np.int32)
    F = {"Gi": I, "Gj": I[:-1].copy(), "Gv": np.ones(n), "IDv": np.full(n, 1e-30),
         "Hi": I.copy(), "Hj": I[:-1].copy(), "Hv": np.ones(n)}
    S = FB.Solver(A, F, variant="afiim", precision="fp32", inner_nmax=3, max_refine=4, reliable=0.0)
    x = np.zeros(n)
    r = S.solve(np.ones(n), x, tol=1e-10, nmax=100)
    assert r["info"] != 0 and r["refine_steps"] <= 4
    S.close()


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
@pytest.mark.parametrize("name,prefix,variant", [("convdiff16_pdfiim", "", "pdfiim"),
                                                 ("poisson128_afiim", "", "afiim"),
                                                 ("convdiff2d48_acifim", "", "acifim")])
def test_reliable_updates_reach_fp64_tolerance(golden, name, prefix, variant, precision):
    """Reliable updates: one FP32 BiCGSTAB whose residual is replaced by the FP64 b - A x; the
    stop is the FP64 test, recomputed here with scipy."""
    g = golden(name)
    A = (g["Ai"], g["Aj"], g["Av"])
    F = {k: v for k, v in sub(g, prefix).items() if k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    S = FB.Solver(A, F, variant=variant, precision=precision, reliable=0.1)
    x = np.zeros(len(g["b"]))
    r = S.solve(g["b"], x, tol=1e-10, nmax=5000)
    tr = relres(A, g["b"], x)
    xo, *_ = O.bicgstab(variant, A, g["b"], F, tol=1e-12, nmax=5000)
    err = np.linalg.norm(x - xo) / np.linalg.norm(xo)
    print(f"{name} {precision} reliable: replacements {r['refine_steps']} its {r['iter']} info {r['info']} "
          f"true relres {tr:.2e} (reported {r['true_relres']:.2e}) err vs FP64 oracle {err:.2e}")
    assert r["info"] == 0
    assert tr <= 1e-10 and abs(tr - r["true_relres"]) <= 1e-3 * tr + 1e-16
    assert r["refine_steps"] >= 1
    assert err <= 1e-6
    S.close()


def test_reliable_updates_same_in_host_loop(golden, monkeypatch):
    """The WHILE graph and the host-relaunched one-iteration graph (with its IF node) run the
    same kernels: the same iterations, replacements and x, bit for bit."""
    g = golden("convdiff16_pdfiim")
    A = (g["Ai"], g["Aj"], g["Av"])
    F = {k: v for k, v in g.items() if k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    out = []
    for mode in (None, "host"):
        if mode:
            monkeypatch.setenv("FIIM_GRAPH", mode)
        S = FB.Solver(A, F, variant="pdfiim", precision="fp32", reliable=0.1)
        x = np.zeros(len(g["b"]))
        r = S.solve(g["b"], x, tol=1e-10, nmax=5000)
        out.append((r["iter"], r["refine_steps"], r["info"], x))
        S.close()
    assert out[0][:3] == out[1][:3]
    assert np.array_equal(out[0][3], out[1][3])


def test_reliable_updates_at_scale():
    """64^3 convection-diffusion, PDFIIM factors: reliable updates (delta 0.1 and the default)
    to 1e-10 in FP32 and BF16 against the FP64 solve to 1e-12, in no more iterations than the
    restarted refinement (reliable = 0)."""
    A = FB.gen_convdiff3d(64, 0.5)
    b = FB.rand_normal(64 ** 3, 20261203)
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    S64 = FB.Solver(A, F, variant="pdfiim")
    x64 = np.zeros(len(b))
    r64 = S64.solve(b, x64, tol=1e-12, nmax=2000)
    assert r64["info"] == 0
    for precision in ("fp32", "bf16"):
        its = {}
        for rel in (0.0, 0.1, None):
            S = FB.Solver(A, F, variant="pdfiim", precision=precision, reliable=rel)
            x = np.zeros(len(b))
            r = S.solve(b, x, tol=1e-10, nmax=5000)
            err = np.linalg.norm(x - x64) / np.linalg.norm(x64)
            print(f"64^3 {precision} reliable={rel}: {r} err vs FP64 {err:.2e}")
            assert r["info"] == 0 and relres(A, b, x) <= 1e-10 and err <= 1e-8
            its[rel] = r["iter"]
            S.close()
        assert its[0.1] <= its[0.0] and its[None] <= its[0.0]
    S64.close()


def test_reliable_updates_end_on_failure():
    """A zero preconditioner (no progress, non-finite scalars) ends the reliable solve with a
    nonzero info within the iteration cap (not a hang); a cap below need gives info 3."""
    A = FB.gen_poisson2d(16)
    n = 256
    I = np.arange(n + 1, dtype=np.int32)
    F = {"Gi": I, "Gj": I[:-1].copy(), "Gv": np.ones(n), "IDv": np.zeros(n),
         "Hi": I.copy(), "Hj": I[:-1].copy(), "Hv": np.ones(n)}
    S = FB.Solver(A, F, variant="afiim", precision="fp32", reliable=0.1, max_refine=4)
    x = np.zeros(n)
    r = S.solve(np.ones(n), x, tol=1e-10, nmax=100)
    assert r["info"] != 0 and r["iter"] <= 101
    S.close()
    g = FB.gen_poisson2d(32)
    Fp = FB.pdfiim_build(g, 0.05, 2, 2, 1, -1, "I", "B")
    S = FB.Solver(g, Fp, variant="pdfiim", precision="fp32", reliable=0.1)
    x = np.zeros(1024)
    r = S.solve(np.ones(1024), x, tol=1e-10, nmax=5)
    assert r["info"] == 3 and r["iter"] == 5
    S.close()


def test_reliable_rejects_bad_delta():
    A = FB.gen_poisson2d(8)
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    for bad in (-0.5, 1.0, 2.0):
        with pytest.raises(FB.FiimError):
            FB.Solver(A, F, variant="pdfiim", precision="fp32", reliable=bad)


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_mixed_diagonal_form_agrees_with_csr_streams(monkeypatch, precision):
    """The mixed solve's inner products read sliced-diagonal copies of the FP32 / BF16 values
    where the matrices allow them (more device memory held); the same solve on the CSR
    streams (FIIM_DIA=0) reaches the same FP64-verified tolerance in about as many
    iterations (the products are the same bits; the fused dot products' trees differ)."""
    A = FB.gen_convdiff3d(48, 0.5)
    n = len(A[0]) - 1
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    b = FB.rand_normal(n, 21)
    out = {}
    for dia in ("1", "0"):
        monkeypatch.setenv("FIIM_DIA", dia)
        S = FB.Solver(A, F, variant="pdfiim", precision=precision)
        x = np.zeros(n)
        r = S.solve(b, x, tol=1e-10, nmax=5000)
        out[dia] = (r, x, S.device_bytes())
        S.close()
    for dia in ("1", "0"):
        r, x, _ = out[dia]
        assert r["info"] == 0 and relres(A, b, x) <= 1e-10
    assert out["1"][2] > out["0"][2]
    assert abs(out["1"][0]["iter"] - out["0"][0]["iter"]) <= 3
