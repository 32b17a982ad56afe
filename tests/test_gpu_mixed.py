"""Mixed precision on B200: FP64 iterative refinement around an FP32 inner BiCGSTAB, with the
factors G, H stored in FP32 or BF16 and D^-1 in FP32.

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
    S = FB.Solver(A, F, variant=variant, precision=precision, inner_tol=1e-5)
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
    solves to 1e-10 against the FP64 GPU solve to 1e-12."""
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
    S = FB.Solver(A, F, variant="afiim", precision="fp32", inner_nmax=3, max_refine=4)
    x = np.zeros(n)
    r = S.solve(np.ones(n), x, tol=1e-10, nmax=100)
    assert r["info"] != 0 and r["refine_steps"] <= 4
    S.close()
