"""Pins of the oracle (CPU only).

The plain-C restatement (oracle/fiim_oracle.c) must reproduce the reference's own solve
bit for bit: against the golden outputs the reference produced (tests/golden), and,
where the reference compiled against the MKL shim is present (oracle/_ref), against
live reference runs on fresh inputs. The MKL shim's arithmetic is checked against
independent numpy/scipy formulations.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import pyoracle as O
import fiim_b200 as FB
from conftest import sub

CASES = [
    ("sherman2", "afiim9e-6_", "afiim", {}, 500),
    ("sherman2", "afiim0.1_", "afiim", {}, 500),
    ("sherman2", "acifim_", "acifim", {"mode": "E", "nr": 2}, 2000),
    ("sherman2", "acifim_", "acifim", {"mode": "C", "nr": 2}, 2000),
    ("sherman2", "pdfiim_", "pdfiim", {}, 1200),
    ("poisson128_afiim", "", "afiim", {}, 1000),
    ("convdiff16_pdfiim", "", "pdfiim", {}, 1200),
    ("convdiff2d48_acifim", "", "acifim", {"mode": "E", "nr": 2}, 2000),
    ("convdiff2d48_acifim", "", "acifim", {"mode": "C", "nr": 2}, 2000),
    ("poisson32_sym_pdfiim", "", "pdfiim", {"issym": True}, 1200),
]


def _result_prefix(name, fprefix, variant, kw):
    if name == "sherman2" and variant == "acifim":
        return f"acifim{kw['mode']}_"
    if name == "convdiff2d48_acifim":
        return f"{kw['mode']}_"
    return fprefix


def csr_of(g, p="A"):
    return g[p + "i"], g[p + "j"], g[p + "v"]


@pytest.mark.parametrize("name,fprefix,variant,kw,nmax", CASES)
def test_restatement_matches_reference_golden(golden, name, fprefix, variant, kw, nmax):
    g = golden(name)
    A, F = csr_of(g), sub(g, fprefix)
    rp = _result_prefix(name, fprefix, variant, kw)
    x, res, it, info = O.bicgstab(variant, A, g["b"], F, tol=1e-8, nmax=nmax, **kw)
    assert it == int(g[rp + "iter"]) and info == int(g[rp + "info"])
    assert res == float(g[rp + "resval"])
    assert np.array_equal(x, g[rp + "x"])


@pytest.mark.parametrize("name,prefix", [("sherman2", "afiim0.1_"), ("poisson128_afiim", ""),
                                         ("convdiff16_pdfiim", ""), ("convdiff2d48_acifim", "")])
def test_restated_products_against_scipy(golden, name, prefix):
    g = golden(name)
    F = sub(g, prefix)
    n = len(g["b"])
    A = sp.csr_matrix((g["Av"], g["Aj"], g["Ai"]), shape=(n, n))
    G = sp.triu(sp.csr_matrix((F["Gv"], F["Gj"], F["Gi"]), shape=(n, n)))
    H = sp.tril(sp.csr_matrix((F["Hv"], F["Hj"], F["Hi"]), shape=(n, n)))
    u = F["u"]
    assert np.allclose(O.csr_mv(*csr_of(g), u), A @ u, rtol=1e-13, atol=1e-13 * np.abs(A @ u).max())
    z = G @ (F["IDv"] * (H @ u))
    assert np.linalg.norm(O.prec_apply(F, u) - z) <= 1e-13 * np.linalg.norm(z)
    assert np.array_equal(O.prec_apply(F, u), F["Mu"])


def test_combined_mode_against_scipy(golden):
    g = golden("convdiff2d48_acifim")
    n = len(g["b"])
    M = lambda p: sp.csr_matrix((g[p + "v"], g[p + "j"], g[p + "i"]), shape=(n, n))
    G, H, L, U = sp.triu(M("G")), sp.tril(M("H")), sp.tril(M("L")), sp.triu(M("U"))
    u, nr = g["u"], 2
    t1 = H @ u
    for _ in range(1, nr):
        t1 = H @ (u - L @ t1) + t1
    t2 = t1 * g["IDv"]
    x = G @ t2
    for _ in range(1, nr):
        x = G @ (t2 - U @ x) + x
    assert np.linalg.norm(g["MuC"] - x) <= 1e-13 * np.linalg.norm(x)


def test_symmetric_products_against_scipy(golden):
    g = golden("poisson32_sym_pdfiim")
    n = len(g["b"])
    Au = sp.csr_matrix((g["Av"], g["Aj"], g["Ai"]), shape=(n, n))
    A = Au + sp.triu(Au, 1).T
    G = sp.triu(sp.csr_matrix((g["Gv"], g["Gj"], g["Gi"]), shape=(n, n)))
    u = g["u"]
    assert np.allclose(g["Au"], A @ u, rtol=1e-13, atol=1e-12)
    z = G @ (g["IDv"] * (G.T @ u))
    assert np.linalg.norm(g["Mu"] - z) <= 1e-13 * np.linalg.norm(z)


def test_golden_reference_solutions_solve_the_systems(golden):
    """Size-independent sanity of the pinned outputs: converged runs have small true residuals."""
    for name, rp in (("poisson128_afiim", ""), ("convdiff16_pdfiim", ""), ("convdiff2d48_acifim", "E_")):
        g = golden(name)
        n = len(g["b"])
        A = sp.csr_matrix((g["Av"], g["Aj"], g["Ai"]), shape=(n, n))
        assert int(g[rp + "info"]) == 0
        assert np.linalg.norm(g["b"] - A @ g[rp + "x"]) <= 1e-7 * np.linalg.norm(g["b"])
    g = golden("poisson128_afiim")
    assert np.abs(g["x"] - 1.0).max() < 1e-5        # b = A*1: the exact solution is all ones


# ----------------------------------------------------------------------- live reference runs
needs_ref = pytest.mark.skipif(not O.have_ref("afiim"), reason="oracle/_ref not built (reference tree absent)")


@needs_ref
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_restatement_matches_live_reference(seed):
    for pkg in ("afiim", "pdfiim", "acifim"):
        O.set_threads(1, pkg)
    rng = np.random.default_rng(seed)
    N = int(rng.integers(12, 24))
    A = FB.gen_convdiff2d(N, float(rng.uniform(0.2, 5)), float(rng.uniform(0, 6.28)), float(rng.uniform(0.1, 1)))
    b = rng.standard_normal(N * N)
    F = O.afiim_build(A, 0.1)
    assert O.ref_solve("afiim", A, b, F)[1:] == O.bicgstab("afiim", A, b, F)[1:]
    Fp = O.pdfiim_build(A, 0.05, 2, 2, 1)
    xr, *r = O.ref_solve("pdfiim", A, b, Fp, nmax=1200)
    xo, *o = O.bicgstab("pdfiim", A, b, Fp, nmax=1200)
    assert r == o and np.array_equal(xr, xo)
    Fc, cerr = O.acifim_build(A, 0.1, 0.05)
    assert cerr == 0
    for mode in "EC":
        xr, *r = O.ref_solve("acifim", A, b, Fc, nmax=2000, mode=mode, nr=3)
        xo, *o = O.bicgstab("acifim", A, b, Fc, nmax=2000, mode=mode, nr=3)
        assert r == o and np.array_equal(xr, xo)


@needs_ref
@pytest.mark.parametrize("blocks", [2, 3, 7])
def test_blocked_restatement_matches_reference_threads(golden, blocks):
    """The restatement's B-block dot products equal the reference's shim on B OpenMP threads."""
    g = golden("sherman2")
    A, F = csr_of(g), sub(g, "afiim0.1_")
    O.set_threads(blocks, "afiim")
    O.set_dot_blocks(blocks)
    try:
        xr, *r = O.ref_solve("afiim", A, g["b"], F)
        xo, *o = O.bicgstab("afiim", A, g["b"], F)
    finally:
        O.set_dot_blocks(1)
        O.set_threads(1, "afiim")
    assert r == o and np.array_equal(xr, xo)


@needs_ref
def test_restatement_matches_live_reference_edge_cases():
    O.set_threads(1, "afiim")
    O.set_threads(1, "acifim")
    A = FB.gen_poisson2d(10)
    n = 100
    F = O.afiim_build(A, 0.1)
    for nmax in (0, 1, 2):
        assert O.ref_solve("afiim", A, FB.model_rhs(A), F, nmax=nmax)[2:] == \
            O.bicgstab("afiim", A, FB.model_rhs(A), F, nmax=nmax)[2:]
    # zero right-hand side: ro = 0, the reference runs to NMAX on NaNs
    r = O.ref_solve("afiim", A, np.zeros(n), F, nmax=7)
    o = O.bicgstab("afiim", A, np.zeros(n), F, nmax=7)
    assert r[2:] == o[2:] == (7, 3) and np.isnan(r[1]) and np.isnan(o[1])
    # stagnation: an unreachable tolerance
    r = O.ref_solve("afiim", A, FB.model_rhs(A), F, tol=1e-30, nmax=500)
    o = O.bicgstab("afiim", A, FB.model_rhs(A), F, tol=1e-30, nmax=500)
    assert r[1:] == o[1:] and r[3] in (1, 2)
    # ACIFIM non-finite alpha guard: skew-symmetric A gives r0.(A r0) = 0
    skew = skew_system(50)
    Fi = identity_factors(50)
    b = np.ones(50)
    Fi_lu = dict(Fi, Li=Fi["Hi"], Lj=Fi["Hj"], Lv=Fi["Hv"], Ui=Fi["Gi"], Uj=Fi["Gj"], Uv=Fi["Gv"])
    r = O.ref_solve("acifim", skew, b, Fi_lu, nmax=30)
    o = O.bicgstab("acifim", skew, b, Fi_lu, nmax=30)
    assert r[2:] == o[2:] == (30, 3)


def skew_system(n):
    """Block diagonal of [[0, 1], [-1, 0]] (zero diagonal stored): with b = 1, b.(A b) = 0 exactly."""
    Ai, Aj, Av = [0], [], []
    for i in range(n):
        ents = ((i, 0.0), (i + 1, 1.0)) if i % 2 == 0 else ((i - 1, -1.0), (i, 0.0))
        for j, v in ents:
            Aj.append(j)
            Av.append(v)
        Ai.append(len(Aj))
    return np.array(Ai, np.int32), np.array(Aj, np.int32), np.array(Av)


def identity_factors(n):
    I = np.arange(n + 1, dtype=np.int32)
    return {"Gi": I, "Gj": I[:-1].copy(), "Gv": np.ones(n), "IDv": np.ones(n),
            "Hi": I.copy(), "Hj": I[:-1].copy(), "Hv": np.ones(n)}


def test_shim_lu_against_numpy():
    """The shim's LAPACKE restatement (used by PDFIIM's construction) solves A x = b and A^T x = b."""
    if not O.have_ref("pdfiim"):
        pytest.skip("oracle/_ref not built")
    import ctypes as C
    lib = O._lib("pdfiim")
    rng = np.random.default_rng(5)
    for m in (1, 2, 5, 17):
        M = rng.standard_normal((m, m)) + np.eye(m) * 0.1
        lu = M.copy()
        piv = np.zeros(m, np.int32)
        assert lib.LAPACKE_dgetrf(101, m, m, lu.ctypes, m, piv.ctypes) == 0
        for trans, ref in ((b"N", M), (b"T", M.T)):
            y = rng.standard_normal(m)
            z = y.copy()
            lib.LAPACKE_dgetrs(101, C.c_char(trans), m, 1, lu.ctypes, m, piv.ctypes, z.ctypes, 1)
            assert np.allclose(z, np.linalg.solve(ref, y), rtol=1e-10, atol=1e-10)
