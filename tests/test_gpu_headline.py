"""The benchmark's own workload against the reference itself (B200 only).

The system is the 3D 7-point upwind convection-diffusion on a 128^3 grid (n = 2,097,152,
nnz = 14,581,760), b ~ N(0,1) from seed 20261203, x0 = 0. The factors are PDFIIM ε 0.05 with
(prefill 2, lfill 2, postfill 1), no warpsize limit, filter 'I' and pattern 'B'. It is checked
against the reference compiled here (oracle/_ref), live, on all host cores:

* factors: the library's host and GPU PDFIIM constructions equal the reference's `pdfiim`
  (PDFIIM/src/parPrec.cpp:95-588) array for array;
* FP64 solve through the reference-facing call fiim_EPBiCGSTAB_pdfiim, with the reference's
  factors: the reference's info; iterations within +-2 of the reference's own counts on
  three thread counts (its dot products are summed per thread, so the count is an envelope);
  resval < tol; x within 10x the reference's own solution spread (floor 1e-9); a true
  residual no worse than 10x the reference's (PDFIIM/src/bicgstab.cpp:80-310);
* mixed precision (FP32 or BF16 factors, FP32 inner BiCGSTAB, FP64 refinement): the
  FP64-verified residual reached, and the relative error against the reference's own FP64
  solution to the same tolerance (1e-8 and 1e-10) below 1e-6 and 1e-7.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import fiim_b200 as FB
import pyoracle as O

pytestmark = pytest.mark.gpu

N, SEED = 128, 20261203
PARAMS = dict(ftol=0.05, prefill=2, lfill=2, postfill=1, warpsize=-1, filttype="I", patt="B")


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def ref128():
    if not O.have_ref("pdfiim"):
        pytest.skip("oracle/_ref (the reference compiled against the MKL shim) is not built")
    A = FB.gen_convdiff3d(N, 0.5)
    b = FB.rand_normal(N ** 3, SEED)
    T = os.cpu_count() or 1
    O.set_threads(T, "pdfiim")
    F = O.pdfiim_build(A, **PARAMS)
    sysr = O.RefPdfiimSystem(A, F)
    runs = {}
    for t in sorted({T, max(1, T // 2), min(T, 3)}, reverse=True):
        O.set_threads(t, "pdfiim")
        x, res, it, info, _ = sysr.run(b, tol=1e-8, nmax=1200)
        runs[t] = (x, res, it, info)
    O.set_threads(T, "pdfiim")
    x10, res10, it10, info10, _ = sysr.run(b, tol=1e-10, nmax=1200)
    sysr.close()
    Asp = sp.csr_matrix((A[2], A[1], A[0]), shape=(N ** 3, N ** 3))
    return {"A": A, "b": b, "F": F, "T": T, "runs": runs, "x10": x10, "it10": it10, "info10": info10, "Asp": Asp}


def true_relres(d, x):
    return float(np.linalg.norm(d["b"] - d["Asp"] @ x) / np.linalg.norm(d["b"]))


@pytest.mark.parametrize("gpu", [False, True])
def test_factors_equal_the_references(ref128, gpu):
    F = FB.pdfiim_build(ref128["A"], **PARAMS, gpu=gpu)
    for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv"):
        assert F[k].dtype == ref128["F"][k].dtype and np.array_equal(F[k], ref128["F"][k]), k


def test_fp64_solve_matches_the_reference(ref128):
    d = ref128
    F = d["F"]
    x = np.zeros(N ** 3)
    resval, it, info = FB.EPBiCGSTAB_pdfiim(d["A"], d["b"], 1e-8, 1200, (F["Gi"], F["Gj"], F["Gv"]), F["IDv"],
                                            (F["Hi"], F["Hj"], F["Hv"]), x)
    xr, resr, itr, infor = d["runs"][d["T"]]
    its = [r[2] for r in d["runs"].values()]
    spread = max(rel(r[0], xr) for r in d["runs"].values())
    print(f"128^3: gpu iter {it} info {info} resval {resval:.3e} | reference iter {itr} (threads "
          f"{sorted(d['runs'])}: {its}) info {infor} | x rel diff {rel(x, xr):.2e}, reference spread {spread:.2e}")
    assert info == infor == 0
    assert all(r[3] == infor for r in d["runs"].values())
    assert min(its) - 2 <= it <= max(its) + 2
    assert resval < 1e-8
    assert rel(x, xr) <= 10 * spread + 1e-9
    assert true_relres(d, x) <= 10 * true_relres(d, xr) + 1e-12


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
@pytest.mark.parametrize("tol,bound", [(1e-8, 1e-6), (1e-10, 1e-7)])
def test_mixed_solve_against_the_references_fp64_solution(ref128, precision, tol, bound):
    """The mixed form's answer against the reference's FP64 solution to the same tolerance."""
    import torch
    d = ref128
    dev = torch.device("cuda:0")
    tA = tuple(torch.from_numpy(a).to(dev) for a in d["A"])
    tF = {k: torch.from_numpy(v).to(dev) for k, v in d["F"].items() if v is not None}
    M = FB.Solver(tA, tF, variant="pdfiim", memory="device", precision=precision, inner_tol=1e-5)
    tb = torch.from_numpy(d["b"]).to(dev)
    tx = torch.zeros_like(tb)
    r = M.solve(tb, tx, tol=tol, nmax=5000)
    M.close()
    x = tx.cpu().numpy()
    xr = d["runs"][d["T"]][0] if tol == 1e-8 else d["x10"]
    err = rel(x, xr)
    tr = true_relres(d, x)
    print(f"{precision} to {tol:g}: inner iterations {r['iter']} in {r['refine_steps']} steps, true relres {tr:.2e} "
          f"(reported {r['true_relres']:.2e}), error vs the reference's FP64 solution {err:.2e}")
    assert r["info"] == 0 and tr <= tol
    assert abs(tr - r["true_relres"]) <= 1e-3 * tr + 1e-15
    assert err <= bound
