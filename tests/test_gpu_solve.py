"""GPU parity of the FP64 solve phase against the oracle (B200 only).

Every check goes through the C-ABI of libfiim_b200.so. Tolerances:
  * SpMV and preconditioner application on the same vector: bit-identical to the
    oracle (each row summed in storage order with rounded products, no FMA), for the
    set-up-free kernel at every lane count and for the solver's tuned kernels.
  * Solves: the same info code; the iteration count within +-2 of the reference's
    rounding envelope (the reference's own counts when only the summation order of its
    dot products changes: the MKL shim's reductions split over 1..8 OpenMP threads,
    recorded in tests/golden); the tolerance reached (resval < tol when converged); the
    solution within 10x the reference's own solution spread, and a true residual no
    worse than 10x the reference's.
"""
import os
import tempfile

import numpy as np
import pytest
import scipy.sparse as sp

import fiim_b200 as FB
import pyoracle as O
from conftest import sub
from test_oracle import identity_factors, skew_system

pytestmark = pytest.mark.gpu

FIXTURE_PRODUCTS = [("sherman2", "afiim9e-6_"), ("sherman2", "afiim0.1_"), ("sherman2", "acifim_"),
                    ("poisson128_afiim", ""), ("convdiff16_pdfiim", ""), ("convdiff2d48_acifim", "")]


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


@pytest.mark.parametrize("name,prefix", FIXTURE_PRODUCTS)
@pytest.mark.parametrize("vec", [0, 2, 4, 8, 16, 32])
def test_spmv_matches_oracle(golden, cuda, name, prefix, vec):
    import torch
    g = golden(name)
    u = sub(g, prefix)["u"]
    Ai, Aj, Av = (_t(g[k], cuda) for k in ("Ai", "Aj", "Av"))
    y = torch.zeros(len(g["b"]), dtype=torch.float64, device=cuda)
    FB.spmv(Ai, Aj, Av, _t(u, cuda), y, vec=vec)
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy(), sub(g, prefix)["Au"])


@pytest.mark.parametrize("name,prefix", FIXTURE_PRODUCTS)
def test_prec_apply_matches_oracle(golden, cuda, name, prefix):
    import torch
    g = golden(name)
    F = sub(g, prefix)
    n = len(g["b"])
    d = {k: _t(F[k], cuda) for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    z = torch.zeros(n, dtype=torch.float64, device=cuda)
    tm = torch.zeros_like(z)
    FB.prec_apply(d["Gi"], d["Gj"], d["Gv"], d["IDv"], d["Hi"], d["Hj"], d["Hv"], _t(F["u"], cuda), z, tm)
    torch.cuda.synchronize()
    assert np.array_equal(z.cpu().numpy(), F["Mu"])


@pytest.mark.parametrize("name,prefix,variant,kw", [
    ("sherman2", "afiim9e-6_", "afiim", {}), ("sherman2", "acifim_", "acifim", {"mode": "C", "nr": 2}),
    ("poisson128_afiim", "", "afiim", {}), ("convdiff16_pdfiim", "", "pdfiim", {}),
    ("convdiff2d48_acifim", "", "acifim", {"mode": "C", "nr": 2}), ("poisson32_sym_pdfiim", "", "pdfiim",
                                                                     {"issym": True})])
@pytest.mark.parametrize("form,cols", [("rows", "narrow"), ("rows", "wide"), ("staged", "wide"), ("warp", "narrow"),
                                       ("warp", "wide")])
def test_solver_products_bit_identical(golden, monkeypatch, name, prefix, variant, kw, form, cols):
    """The solver's tuned CSR-stream kernels (streams through registers, with 16-bit or 32-bit
    column streams, or by bulk copies) reproduce the oracle's A x and M x exactly."""
    monkeypatch.setenv("FIIM_SPMV", form)
    monkeypatch.setenv("FIIM_COLS", cols)
    g = golden(name)
    F = sub(g, prefix)
    S = FB.Solver((g["Ai"], g["Aj"], g["Av"]), F, variant=variant, autotune=True, **kw)
    n = len(g["b"])
    y = S.apply(F["u"], np.zeros(n), op="A")
    assert np.array_equal(y, F["Au"])
    z = S.apply(F["u"], np.zeros(n), op="M")
    assert np.array_equal(z, F["MuC"] if kw.get("mode") == "C" else F["Mu"])
    S.close()


def dia_bytes(rp, ci):
    """Bytes of the sliced-diagonal copy of a CSR matrix (slices of 32 rows, 8 bytes per slot
    of each slice's diagonals, a record of 16 or 32 ints per slice), or None when a row is
    unsorted or a slice has more than 28 diagonals."""
    n = len(rp) - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    if np.any((np.diff(ci) <= 0) & (np.diff(rows) == 0)):
        return None
    d = ci.astype(np.int64) - rows
    key = np.unique((rows // 32) * (4 * n) + (d + 2 * n))
    per = np.bincount(key // (4 * n), minlength=(n + 31) // 32)
    if per.max() > 28:
        return None
    nd = int(per.sum())
    return 8.0 * 32 * nd + 4.0 * (16 if per.max() <= 12 else 32) * len(per)


@pytest.mark.parametrize("name,prefix,variant", [("sherman2", "afiim9e-6_", "afiim"), ("poisson128_afiim", "", "afiim"),
                                                 ("convdiff16_pdfiim", "", "pdfiim"),
                                                 ("convdiff2d48_acifim", "", "acifim")])
def test_dia_form_products_bit_identical(golden, name, prefix, variant):
    """By default the solver reads the sliced-diagonal copy of each matrix whose rows allow it
    (form 3) and the CSR streams otherwise; A x and M x equal the oracle's bit for bit."""
    g = golden(name)
    F = sub(g, prefix)
    A = (g["Ai"], g["Aj"], g["Av"])
    S = FB.Solver(A, F, variant=variant)
    n = len(g["b"])
    for which, (rp, ci) in enumerate([(A[0], A[1]), (F["Gi"], F["Gj"]), (F["Hi"], F["Hj"])]):
        db = dia_bytes(rp, ci)
        nnz = len(ci)
        form = S.spmv_shape(which)[1]
        if db is None or db >= nnz * 12 + 4 * (n + 1):
            assert form != 3
        elif db < nnz * 10 + 4 * (n + 1):
            assert form == 3
    assert np.array_equal(S.apply(F["u"], np.zeros(n), op="A"), F["Au"])
    assert np.array_equal(S.apply(F["u"], np.zeros(n), op="M"), F["Mu"])
    S.close()


def test_dia_form_on_the_headline_structure():
    """The 3D convection-diffusion matrix and its PDFIIM factors take the sliced-diagonal form;
    A x and M x equal the CSR streams' (FIIM_SPMV=rows) bit for bit. The solves differ only
    through the fused dot products, whose summation tree follows the launch shape."""
    A = FB.gen_convdiff3d(48, 0.5)
    n = len(A[0]) - 1
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    b = FB.rand_normal(n, 5)
    u = FB.rand_normal(n, 6)
    out = {}
    for form in (None, "rows"):
        env = os.environ.pop("FIIM_SPMV", None)
        if form:
            os.environ["FIIM_SPMV"] = form
        try:
            S = FB.Solver(A, F, variant="pdfiim")
            forms = [S.spmv_shape(w)[1] for w in range(3)]
            x = np.zeros(n)
            r = S.solve(b, x, tol=1e-10, nmax=500)
            out[form] = (forms, S.apply(u, np.zeros(n), op="A"), S.apply(u, np.zeros(n), op="M"), x, r["iter"])
            S.close()
        finally:
            os.environ.pop("FIIM_SPMV", None)
            if env is not None:
                os.environ["FIIM_SPMV"] = env
    assert out[None][0] == [3, 3, 3] and 3 not in out["rows"][0]
    for k in (1, 2):
        assert np.array_equal(out[None][k], out["rows"][k])
    assert abs(out[None][4] - out["rows"][4]) <= 2
    assert np.linalg.norm(out[None][3] - out["rows"][3]) <= 1e-7 * np.linalg.norm(out["rows"][3])


def test_dia_form_refused_for_unsorted_rows_and_the_padding_pattern():
    """Rows not sorted by column, and an entry holding the padding's bit pattern, keep the CSR
    streams; the products stay the oracle's."""
    A = FB.gen_convdiff3d(40, 0.5)
    n = len(A[0]) - 1
    F = identity_factors(n)
    u = FB.rand_normal(n, 9)
    Av = A[2].copy()
    Aj = A[1].copy()
    e = A[0][(5 * 40 + 5) * 40 + 5]          # the first entry of an interior row (7 entries)
    Aj[[e, e + 1]] = Aj[[e + 1, e]]
    Av[[e, e + 1]] = Av[[e + 1, e]]
    S = FB.Solver((A[0], Aj, Av), F)
    assert S.spmv_shape(0)[1] != 3
    assert np.array_equal(S.apply(u, np.zeros(n), op="A"), O.csr_mv(A[0], Aj, Av, u))
    S.close()
    Av = A[2].copy()
    Av[500] = np.frombuffer(np.uint64(0xFFF7D1A6B00C5A1D).tobytes(), dtype=np.float64)[0]
    S = FB.Solver((A[0], A[1], Av), F)
    assert S.spmv_shape(0)[1] != 3
    y = S.apply(u, np.zeros(n), op="A")
    ref = O.csr_mv(A[0], A[1], Av, u)
    assert np.array_equal(np.isnan(y), np.isnan(ref)) and np.array_equal(y[~np.isnan(y)], ref[~np.isnan(ref)])
    S.close()


def test_dropin_reload_replaces_diagonal_values():
    """A drop-in call with new values in the same structure re-places them in the existing
    sliced-diagonal copy: the result equals a fresh solver's bit for bit."""
    A = FB.gen_convdiff3d(40, 0.5)
    n = len(A[0]) - 1
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    G, H = (F["Gi"], F["Gj"], F["Gv"]), (F["Hi"], F["Hj"], F["Hv"])
    b = FB.rand_normal(n, 13)
    prev = FB.dropin_cache(True)
    try:
        for scale in (1.0, 1.25):
            AA = (A[0], A[1], A[2] * scale)
            x = np.zeros(n)
            r = FB.EPBiCGSTAB_pdfiim(AA, b, 1e-10, 500, G, F["IDv"], H, x)
            S = FB.Solver(AA, F, variant="pdfiim")
            assert S.spmv_shape(0)[1] == 3
            y = np.zeros(n)
            r1 = S.solve(b, y, tol=1e-10, nmax=500)
            S.close()
            assert np.array_equal(x, y) and r[1] == r1["iter"]
    finally:
        FB.dropin_cache(prev)


def test_dropin_reload_takes_each_calls_b_and_x0():
    """With the device-copy reuse off every drop-in call uploads the system again, with its
    b and x0 copied ahead of the matrices. Calls with other right-hand sides and nonzero
    initial guesses, over new values in the same structure and then the same values, each
    equal a fresh solver's result bit for bit."""
    A = FB.gen_convdiff3d(40, 0.5)
    n = len(A[0]) - 1
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    G, H = (F["Gi"], F["Gj"], F["Gv"]), (F["Hi"], F["Hj"], F["Hv"])
    prev = FB.dropin_cache(False)
    try:
        for k, scale in enumerate((1.0, 1.0, 0.8, 0.8)):
            AA = (A[0], A[1], A[2] * scale)
            b = FB.rand_normal(n, 101 + k)
            x0 = 0.01 * k * FB.rand_normal(n, 201 + k)
            x = x0.copy()
            r = FB.EPBiCGSTAB_pdfiim(AA, b, 1e-10, 500, G, F["IDv"], H, x)
            S = FB.Solver(AA, F, variant="pdfiim")
            y = x0.copy()
            r1 = S.solve(b, y, tol=1e-10, nmax=500)
            S.close()
            assert r[2] == 0 and np.array_equal(x, y) and r[1] == r1["iter"], k
    finally:
        FB.dropin_cache(prev)


def test_dropin_reload_value_with_padding_pattern():
    """A reload whose H holds the sliced-diagonal padding pattern as a value (a NaN) gives H's
    copy up for the CSR streams, as a fresh solver does at set-up. The calls before and
    after it, with ordinary values in the same structure, equal a fresh solver's results bit
    for bit (the pattern's call NaN for NaN)."""
    A = FB.gen_convdiff3d(40, 0.5)   # 64,000 rows: the graph path, whose products read the copies
    n = len(A[0]) - 1
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    G = (F["Gi"], F["Gj"], F["Gv"])
    b = FB.rand_normal(n, 17)
    pad = np.array([0xFFF7D1A6B00C5A1D], dtype=np.uint64).view(np.float64)[0]
    prev = FB.dropin_cache(False)
    try:
        for k in range(3):
            Hv = F["Hv"].copy()
            if k == 1:
                Hv[len(Hv) // 2] = pad
            H = (F["Hi"], F["Hj"], Hv)
            x = np.zeros(n)
            r = FB.EPBiCGSTAB_pdfiim(A, b, 1e-10, 40, G, F["IDv"], H, x)
            FF = dict(F, Hv=Hv)
            S = FB.Solver(A, FF, variant="pdfiim")
            form = S.spmv_shape(2)[1]
            assert (form != 3) if k == 1 else (form == 3), k
            y = np.zeros(n)
            r1 = S.solve(b, y, tol=1e-10, nmax=40)
            S.close()
            assert np.array_equal(x, y, equal_nan=True) and r[1] == r1["iter"], k
            assert np.isfinite(x).all() == (k != 1), k
    finally:
        FB.dropin_cache(prev)


@pytest.mark.parametrize("form", [None, "staged", "warp"])
@pytest.mark.parametrize("long_len", [0, 2046, 2047, 2048, 2500])
def test_solver_spmv_random_rows(monkeypatch, long_len, form):
    """Random columns over the whole matrix, row blocks that start at odd entries, and a
    few rows of about the row-block size (2048 entries for this mean row length): rows
    that fill a block exactly, one entry short of it, or exceed it. A x through the
    solver's row blocks equals the oracle's bit for bit, in the default form and in the
    form that copies 16-byte aligned windows by bulk copies."""
    rng = np.random.default_rng(long_len)
    n = 200000 if long_len == 0 else 20000
    lens = rng.integers(1, 10, n)
    rows, cols = [], []
    for i, k in enumerate(lens):
        if long_len and i % 1700 == 7:
            k = long_len
        rows.append(np.full(k, i))
        cols.append(rng.choice(n, k, replace=False) if k > 64 else rng.integers(0, n, k))
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    M = sp.csr_matrix((rng.uniform(-1, 1, rows.size), (rows, cols)), shape=(n, n))
    M.sum_duplicates()
    M.sort_indices()
    A = (M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data)
    if long_len:
        assert (np.diff(A[0]) == long_len).sum() == 12
    u = rng.standard_normal(n)
    if form:
        monkeypatch.setenv("FIIM_SPMV", form)
    S = FB.Solver(A, identity_factors(n), autotune=form is not None)
    if form is None:
        assert S.spmv_shape(0) == (2048, 0)
    y = S.apply(u, np.zeros(n), op="A")
    S.close()
    assert np.array_equal(y, O.csr_mv(*A, u))


@pytest.mark.parametrize("spread", [60000, 70000, 400000])
def test_solver_spmv_column_spans(spread):
    """Row blocks whose columns span more than 65,536 keep 32-bit columns (the matrix falls
    back as a whole); narrower spans use 16-bit offsets from a per-block base. Either way A x
    equals the oracle's bit for bit."""
    rng = np.random.default_rng(spread)
    n = 200000
    rows = np.repeat(np.arange(n), 6)
    cols = np.clip(rows + rng.integers(-spread // 2, spread // 2 + 1, rows.size), 0, n - 1)
    M = sp.csr_matrix((rng.uniform(-1, 1, rows.size), (rows, cols)), shape=(n, n)) + sp.eye(n) * 8
    M.sum_duplicates()
    M.sort_indices()
    A = (M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data)
    u = rng.standard_normal(n)
    S = FB.Solver(A, identity_factors(n))
    y = S.apply(u, np.zeros(n), op="A")
    S.close()
    assert np.array_equal(y, O.csr_mv(*A, u))


@pytest.mark.parametrize("name,variant", [("poisson128_afiim", "afiim"), ("convdiff16_pdfiim", "pdfiim"),
                                          ("sherman2", "pdfiim")])
def test_one_launch_solve_matches_graph(golden, monkeypatch, name, variant):
    """Small systems solve as one cooperative launch (grid barriers between the phases). The
    products and updates are the launched kernels' arithmetic; only the dot products' tree
    differs, so it ends like the WHILE-graph solve: same info, iterations within +-2, x
    within the reference's own spread."""
    g = golden(name)
    prefix = "pdfiim_" if name == "sherman2" else ""
    F = {k: g[prefix + k] for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    A = (g["Ai"], g["Aj"], g["Av"])
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("FIIM_PERSIST", mode)
        S = FB.Solver(A, F, variant=variant)
        assert S.mode() == (2 if mode == "1" else 0)
        x = np.zeros(len(g["b"]))
        r = S.solve(g["b"], x, tol=1e-8, nmax=1200)
        S.close()
        out[mode] = (x, r)
    (xp, rp), (xg, rg) = out["1"], out["0"]
    lo, hi = (int(v) for v in g[prefix + "iter_env"])
    print(f"{name}: one launch {rp['iter']} iterations, graph {rg['iter']}, envelope [{lo},{hi}]")
    assert rp["info"] == rg["info"]
    if rp["info"] == 0:
        assert lo - 2 <= rp["iter"] <= hi + 2 and rp["true_relres"] < 1e-7
        spread = max(float(g[prefix + "x_spread"]), 1e-9)
        assert np.linalg.norm(xp - xg) / np.linalg.norm(xg) <= 10 * spread
    assert rp["launches"] == 1


def test_one_launch_barrier_wait_is_bounded(monkeypatch):
    """A grid barrier that can never complete (test hook) ends the solve with FIIM_ETIMEOUT
    after the wait limit instead of hanging; the next solve on the same handle is correct."""
    monkeypatch.setenv("FIIM_PERSIST", "1")
    A = FB.gen_poisson2d(64)
    n = 64 * 64
    F = FB.pdfiim_build(A, 0.05, 1, 1, 1)
    b = FB.rand_normal(n, 9)
    S = FB.Solver(A, F, variant="pdfiim")
    assert S.mode() == 2
    x0 = np.zeros(n)
    r0 = S.solve(b, x0, tol=1e-8, nmax=500)
    S.set_wait_limit(20000)
    S.test_stall()
    x = np.zeros(n)
    with pytest.raises(FB.FiimError) as e:
        S.solve(b, x, tol=1e-8, nmax=500)
    assert e.value.rc == FB.FIIM_ETIMEOUT and "barrier" in str(e.value)
    S.set_wait_limit(1 << 21)
    x2 = np.zeros(n)
    r2 = S.solve(b, x2, tol=1e-8, nmax=500)
    S.close()
    assert np.array_equal(x2, x0) and r2["iter"] == r0["iter"] and r2["info"] == 0


def test_prec_apply_ignores_entries_outside_triangles(cuda):
    """MKL TRIANGULAR descriptors read one triangle (AFIIM/src/bicgstab.cpp:140-147)."""
    import torch
    rng = np.random.default_rng(3)
    n = 300
    M = sp.random(n, n, density=0.05, random_state=4, format="csr") + sp.eye(n)
    M.sort_indices()
    F = {"Gi": M.indptr, "Gj": M.indices, "Gv": M.data, "IDv": rng.uniform(0.5, 2, n),
         "Hi": M.indptr, "Hj": M.indices, "Hv": M.data}
    u = rng.standard_normal(n)
    want = O.prec_apply(F, u)
    d = {k: _t(np.asarray(F[k], np.int32 if k[1] in "ij" else np.float64), cuda) for k in F}
    z = torch.zeros(n, dtype=torch.float64, device=cuda)
    FB.prec_apply(d["Gi"], d["Gj"], d["Gv"], d["IDv"], d["Hi"], d["Hj"], d["Hv"], _t(u, cuda), z,
                  torch.zeros_like(z))
    torch.cuda.synchronize()
    assert np.array_equal(z.cpu().numpy(), want)
    # the solver path filters the triangles at upload and must agree too
    S = FB.Solver((M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data), {k: np.asarray(v) for k, v in F.items()})
    assert np.array_equal(S.apply(u, np.zeros(n), op="M"), want)
    S.close()


SOLVES = [
    ("sherman2", "afiim9e-6_", "afiim9e-6_", "afiim", {}, 500),
    ("sherman2", "afiim0.1_", "afiim0.1_", "afiim", {}, 500),
    ("sherman2", "acifim_", "acifimE_", "acifim", {"mode": "E", "nr": 2}, 2000),
    ("sherman2", "acifim_", "acifimC_", "acifim", {"mode": "C", "nr": 2}, 2000),
    ("sherman2", "pdfiim_", "pdfiim_", "pdfiim", {}, 1200),
    ("poisson128_afiim", "", "", "afiim", {}, 1000),
    ("convdiff16_pdfiim", "", "", "pdfiim", {}, 1200),
    ("convdiff2d48_acifim", "", "E_", "acifim", {"mode": "E", "nr": 2}, 2000),
    ("convdiff2d48_acifim", "", "C_", "acifim", {"mode": "C", "nr": 2}, 2000),
    ("poisson32_sym_pdfiim", "", "", "pdfiim", {"issym": True}, 1200),
]


def dropin(variant, g, F, nmax, x, tol=1e-8, mode="E", nr=1, issym=False):
    n = len(g["b"])
    if variant == "afiim":
        return FB.EPBiCGSTAB(n, g["Av"], g["Aj"], g["Ai"], g["b"], tol, nmax, F["Gv"], F["Gj"], F["Gi"], F["IDv"],
                             F["Hv"], F["Hj"], F["Hi"], x)
    if variant == "pdfiim":
        H = None if issym else (F["Hi"], F["Hj"], F["Hv"])
        return FB.EPBiCGSTAB_pdfiim((g["Ai"], g["Aj"], g["Av"]), g["b"], tol, nmax, (F["Gi"], F["Gj"], F["Gv"]),
                                    F["IDv"], H, x, issym=issym)
    return FB.PBiCGSTAB(n, g["Av"], g["Aj"], g["Ai"], g["b"], tol, nmax, F["Gv"], F["Gj"], F["Gi"], F["IDv"],
                        F["Hv"], F["Hj"], F["Hi"], F.get("Lv"), F.get("Lj"), F.get("Li"), F.get("Uv"), F.get("Uj"),
                        F.get("Ui"), nr, mode, x)


def true_relres(g, x):
    n = len(g["b"])
    A = sp.csr_matrix((g["Av"], g["Aj"], g["Ai"]), shape=(n, n))
    if "sym" in g["meta"]["system"].lower() or "SYMMETRIC" in g["meta"]["system"]:
        A = A + sp.triu(A, 1).T
    return np.linalg.norm(g["b"] - A @ x) / np.linalg.norm(g["b"])


@pytest.mark.parametrize("name,fprefix,rprefix,variant,kw,nmax", SOLVES)
def test_dropin_solve_matches_reference(golden, name, fprefix, rprefix, variant, kw, nmax):
    """Same info; iterations within +-2 of the reference's rounding envelope (its own counts
    when only the summation order of its reductions changes, OpenMP 1..8 threads); the
    tolerance reached; x within the reference's own solution spread (x 10, floor 1e-9) and
    a true residual no worse than 10x the reference's."""
    g = golden(name)
    F = sub(g, fprefix)
    x = np.zeros(len(g["b"]))
    resval, it, info = dropin(variant, g, F, nmax, x, **kw)
    ref_it, ref_info = int(g[rprefix + "iter"]), int(g[rprefix + "info"])
    lo, hi = (int(v) for v in g[rprefix + "iter_env"])
    dx = rel(x, g[rprefix + "x"])
    print(f"{name}/{rprefix or variant}: gpu iter {it} info {info} resval {resval:.3e} | ref iter {ref_it} "
          f"envelope [{lo},{hi}] info {ref_info} | x rel diff {dx:.2e} (ref spread {float(g[rprefix + 'x_spread']):.2e})")
    assert info == ref_info
    assert lo - 2 <= it <= hi + 2
    if ref_info == 0:
        assert resval < 1e-8
    assert dx <= 10 * float(g[rprefix + "x_spread"]) + 1e-9
    assert true_relres(g, x) <= 10 * true_relres(g, g[rprefix + "x"]) + 1e-12


@pytest.mark.parametrize("form", ["rows", "staged", "warp", "dia"])
def test_solver_forms_agree_on_convdiff64(monkeypatch, form):
    """A 64^3 solve takes the same iterations and (to rounding) the same x with either SpMV form."""
    monkeypatch.setenv("FIIM_SPMV", form)
    A = FB.gen_convdiff3d(64, 0.5)
    b = FB.rand_normal(64 ** 3, 20261203)
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    S = FB.Solver(A, F, variant="pdfiim", autotune=True)
    x = np.zeros(64 ** 3)
    r = S.solve(b, x, tol=1e-8, nmax=1200)
    S.close()
    # The products are the same bits in both forms; the fused dot products are summed in a
    # launch-shape-dependent tree, so x may differ in its last bits.
    ref = np.load(_forms_cache()) if os.path.exists(_forms_cache()) else None
    if ref is None:
        np.save(_forms_cache(), x)
    else:
        assert np.linalg.norm(ref - x) <= 1e-12 * np.linalg.norm(ref)
    assert r["info"] == 0 and r["iter"] == 58


def _forms_cache():
    return os.path.join(tempfile.gettempdir(), f"fiim_forms_{os.getpid()}.npy")


def test_dropin_reload_follows_row_structure():
    """A drop-in call with a system of the same size and entry count but other row offsets
    rebuilds the row blocks: its result equals a fresh solver's bit for bit."""
    A = FB.gen_convdiff3d(12, 0.5)
    n = len(A[0]) - 1
    M = sp.csr_matrix((A[2], A[1], A[0]), shape=(n, n))
    P = sp.eye(n, format="csr")[np.random.default_rng(5).permutation(n)]
    M2 = (P @ M @ P.T).tocsr()
    M2.sort_indices()
    A2 = (M2.indptr.astype(np.int32), M2.indices.astype(np.int32), M2.data.copy())
    assert len(A2[1]) == len(A[1]) and not np.array_equal(A2[0], A[0])
    F = identity_factors(n)
    G, H = (F["Gi"], F["Gj"], F["Gv"]), (F["Hi"], F["Hj"], F["Hv"])
    b = FB.rand_normal(n, 3)
    prev = FB.dropin_cache(False)
    try:
        for AA in (A, A2):
            x = np.zeros(n)
            r = FB.EPBiCGSTAB_pdfiim(AA, b, 1e-10, 500, G, F["IDv"], H, x)
            S = FB.Solver(AA, F, variant="pdfiim")
            y = np.zeros(n)
            r1 = S.solve(b, y, tol=1e-10, nmax=500)
            S.close()
            assert np.array_equal(x, y) and r[1] == r1["iter"]
    finally:
        FB.dropin_cache(prev)


def test_dropin_reload_follows_column_indices():
    """A drop-in call with the same row offsets as the previous one but other column indices
    rebuilds the narrow column stream: its result equals a fresh solver's bit for bit. The
    system (64,000 rows) takes the graph path, whose products read that stream."""
    A = FB.gen_convdiff3d(40, 0.5)
    n = len(A[0]) - 1
    A2 = (A[0].copy(), ((A[1].astype(np.int64) + 977) % n).astype(np.int32), A[2].copy())
    assert np.array_equal(A2[0], A[0]) and not np.array_equal(A2[1], A[1])
    F = identity_factors(n)
    G, H = (F["Gi"], F["Gj"], F["Gv"]), (F["Hi"], F["Hj"], F["Hv"])
    b = FB.rand_normal(n, 11)
    prev = FB.dropin_cache(False)
    try:
        for AA in (A, A2, A):
            x = np.zeros(n)
            r = FB.EPBiCGSTAB_pdfiim(AA, b, 1e-14, 25, G, F["IDv"], H, x)
            S = FB.Solver(AA, F, variant="pdfiim")
            assert S.mode() in (0, 1)
            y = np.zeros(n)
            r1 = S.solve(b, y, tol=1e-14, nmax=25)
            S.close()
            assert np.array_equal(x, y) and r[1] == r1["iter"]
    finally:
        FB.dropin_cache(prev)


def test_dropin_cache_follows_array_contents():
    """Repeated drop-in calls reuse the device copies only while every matrix array keeps
    its address, size and contents: a value changed in place is uploaded again, and the
    result equals a call that uploads everything."""
    A = FB.gen_convdiff3d(16, 0.5)
    n = len(A[0]) - 1
    b = FB.rand_normal(n, 7)
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    G, H = (F["Gi"], F["Gj"], F["Gv"]), (F["Hi"], F["Hj"], F["Hv"])

    def run():
        x = np.zeros(n)
        r = FB.EPBiCGSTAB_pdfiim(A, b, 1e-10, 500, G, F["IDv"], H, x)
        return x, r

    prev = FB.dropin_cache(True)
    try:
        x1, r1 = run()
        x2, r2 = run()          # same arrays: no upload
        assert np.array_equal(x1, x2) and r1 == r2
        A[2][5] *= 1.5          # changed in place: same address and size
        F["Hv"][7] *= 0.5
        x3, r3 = run()
        FB.dropin_cache(False)
        x4, r4 = run()          # everything uploaded
        assert np.array_equal(x3, x4) and r3 == r4
        assert not np.array_equal(x3, x1)
    finally:
        FB.dropin_cache(prev)


@pytest.mark.parametrize("memory", ["host", "device"])
def test_handle_api_matches_dropin(golden, cuda, memory):
    import torch
    g = golden("poisson128_afiim")
    F = {k: g[k] for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    A = (g["Ai"], g["Aj"], g["Av"])
    x0 = np.zeros(len(g["b"]))
    r_drop = FB.EPBiCGSTAB(len(g["b"]), g["Av"], g["Aj"], g["Ai"], g["b"], 1e-8, 1000, F["Gv"], F["Gj"], F["Gi"],
                           F["IDv"], F["Hv"], F["Hj"], F["Hi"], x0)
    if memory == "device":
        A = tuple(_t(a, cuda) for a in A)
        F = {k: _t(v, cuda) for k, v in F.items()}
        b, x = _t(g["b"], cuda), torch.zeros(len(g["b"]), dtype=torch.float64, device=cuda)
    else:
        b, x = g["b"], np.zeros(len(g["b"]))
    S = FB.Solver(A, F, variant="afiim", memory=memory)
    r = S.solve(b, x, tol=1e-8, nmax=1000)
    xs = x.cpu().numpy() if memory == "device" else x
    assert (r["resval"], r["iter"], r["info"]) == r_drop
    assert np.array_equal(xs, x0)
    assert r["true_relres"] < 1e-7 and r["device_ms"] > 0
    # the WHILE graph launches 9 kernels per iteration; a one-launch or one-cluster solve launches 1
    assert r["launches"] > r["iter"] * 9 if S.mode() not in (2, 3) else r["launches"] == 1
    S.close()


def test_repeated_solves_are_bitwise_deterministic(golden):
    g = golden("convdiff16_pdfiim")
    F = {k: g[k] for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    S = FB.Solver((g["Ai"], g["Aj"], g["Av"]), F, variant="pdfiim")
    xs = []
    for _ in range(3):
        x = np.zeros(len(g["b"]))
        r = S.solve(g["b"], x, tol=1e-8, nmax=1200)
        xs.append((x, r["resval"], r["iter"]))
    assert all(np.array_equal(xs[0][0], o[0]) and xs[0][1:] == o[1:] for o in xs[1:])


def test_edge_cases_match_oracle(golden):
    g = golden("poisson128_afiim")
    A = (g["Ai"], g["Aj"], g["Av"])
    F = {k: g[k] for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    S = FB.Solver(A, F, variant="afiim")
    n = len(g["b"])
    for nmax in (0, 1, 2, 5):
        x = np.zeros(n)
        r = S.solve(g["b"], x, tol=1e-8, nmax=nmax)
        xo, res, it, info = O.bicgstab("afiim", A, g["b"], F, tol=1e-8, nmax=nmax)
        assert (r["iter"], r["info"]) == (it, info)
        assert rel(x, xo) <= 1e-10 if nmax > 0 else np.array_equal(x, xo)
    # nonzero initial guess
    x0 = FB.rand_normal(n, 11)
    x = x0.copy()
    r = S.solve(g["b"], x, tol=1e-8, nmax=1000)
    xo, res, it, info = O.bicgstab("afiim", A, g["b"], F, tol=1e-8, nmax=1000, x0=x0)
    assert r["info"] == info == 0 and abs(r["iter"] - it) <= 2
    # zero right-hand side: ro = 0; the reference runs to NMAX on NaNs
    x = np.zeros(n)
    r = S.solve(np.zeros(n), x, tol=1e-8, nmax=6)
    assert (r["iter"], r["info"]) == (6, 3) and np.isnan(r["resval"])
    # unreachable tolerance: the oracle's stagnation / divergence exit
    x = np.zeros(n)
    r = S.solve(g["b"], x, tol=1e-30, nmax=1000)
    xo, res, it, info = O.bicgstab("afiim", A, g["b"], F, tol=1e-30, nmax=1000)
    assert r["info"] == info and info in (1, 2)
    S.close()


def test_acifim_nonfinite_alpha_guard():
    """ACIFIM/src/bicgstab.cpp:208-213: alpha = m1 / 0 ends the solve with iter = NMAX, info 3."""
    A = skew_system(64)
    F = identity_factors(64)
    F.update(Li=F["Hi"], Lj=F["Hj"], Lv=F["Hv"], Ui=F["Gi"], Uj=F["Gj"], Uv=F["Gv"])
    b = np.ones(64)
    for mode in "EC":
        x = np.zeros(64)
        res, it, info = FB.PBiCGSTAB(64, A[2], A[1], A[0], b, 1e-8, 25, F["Gv"], F["Gj"], F["Gi"], F["IDv"], F["Hv"],
                                     F["Hj"], F["Hi"], F["Lv"], F["Lj"], F["Li"], F["Uv"], F["Uj"], F["Ui"], 2, mode, x)
        xo, reso, ito, infoo = O.bicgstab("acifim", A, b, F, nmax=25, mode=mode, nr=2)
        assert (it, info) == (ito, infoo) == (25, 3)
        assert not x.any()


def test_convdiff64_host_factors_match_oracle():
    """The 128^3 workload's stencil at 64^3 with the product's own PDFIIM factors."""
    A = FB.gen_convdiff3d(64, 0.5)
    b = FB.rand_normal(64 ** 3, 20261203)
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    x = np.zeros(64 ** 3)
    S = FB.Solver(A, F, variant="pdfiim")
    r = S.solve(b, x, tol=1e-8, nmax=1200)
    xo, reso, ito, infoo = O.bicgstab("pdfiim", A, b, F, tol=1e-8, nmax=1200)
    print("64^3:", r, "oracle", ito, infoo, reso)
    assert r["info"] == infoo == 0 and abs(r["iter"] - ito) <= 2
    assert r["true_relres"] < 1e-7 and rel(x, xo) < 1e-6
    tr = np.linalg.norm(b - sp.csr_matrix((A[2], A[1], A[0])) @ x) / np.linalg.norm(b)
    assert abs(tr - r["true_relres"]) <= 1e-3 * tr
    S.close()


@pytest.mark.parametrize("long_len", [254, 255, 256, 257, 600])
def test_solver_warp_form_rows_about_its_block_size(monkeypatch, long_len):
    """The warp-block form (blocks of at most 32 rows and 255 entries): rows that fill a
    block, one entry short of it, or need the long-row path. A x equals the oracle's bit
    for bit."""
    rng = np.random.default_rng(long_len)
    n = 30000
    lens = rng.integers(1, 12, n)
    rows, cols = [], []
    for i, k in enumerate(lens):
        if i % 997 == 3:
            k = long_len
        rows.append(np.full(k, i))
        cols.append(rng.choice(n, k, replace=False))
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    M = sp.csr_matrix((rng.uniform(-1, 1, rows.size), (rows, cols)), shape=(n, n))
    M.sort_indices()
    A = (M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data)
    u = rng.standard_normal(n)
    monkeypatch.setenv("FIIM_SPMV", "warp")
    S = FB.Solver(A, identity_factors(n))
    assert S.spmv_shape(0) == (256, 2)
    y = S.apply(u, np.zeros(n), op="A")
    S.close()
    assert np.array_equal(y, O.csr_mv(A[0], A[1], A[2], u))


@pytest.mark.parametrize("name,variant", [("poisson128_afiim", "afiim"), ("convdiff16_pdfiim", "pdfiim"),
                                          ("sherman2", "pdfiim"), ("convdiff2d48_acifim", "acifim")])
def test_cluster_solve_matches_graph(golden, monkeypatch, name, variant):
    """Small systems solve in one thread-block cluster, vectors in the CTAs' shared memory and
    gathered across it. The products and updates are the launched kernels' arithmetic; only
    the dot products' tree differs, so it ends like the WHILE-graph solve: same info,
    iterations within +-2 of the reference's envelope, x within the reference's own spread."""
    g = golden(name)
    prefix = "pdfiim_" if name == "sherman2" else ""
    F = {k: g[prefix + k] for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    A = (g["Ai"], g["Aj"], g["Av"])
    env_prefix = "E_" if name == "convdiff2d48_acifim" else prefix
    out = {}
    for mode in ("cluster", "0"):
        monkeypatch.setenv("FIIM_PERSIST", mode)
        S = FB.Solver(A, F, variant=variant)
        assert S.mode() == (3 if mode == "cluster" else 0)
        x = np.zeros(len(g["b"]))
        r = S.solve(g["b"], x, tol=1e-8, nmax=2000)
        S.close()
        out[mode] = (x, r)
    (xc, rc), (xg, rg) = out["cluster"], out["0"]
    lo, hi = (int(v) for v in g[env_prefix + "iter_env"])
    print(f"{name}: cluster {rc['iter']} iterations, graph {rg['iter']}, envelope [{lo},{hi}]")
    assert rc["info"] == rg["info"] == int(g[env_prefix + "info"])
    if rc["info"] == 0:
        assert lo - 2 <= rc["iter"] <= hi + 2 and rc["resval"] < 1e-8
        spread = max(float(g[env_prefix + "x_spread"]), 1e-9)
        assert np.linalg.norm(xc - xg) / np.linalg.norm(xg) <= 10 * spread
        assert abs(rc["true_relres"] - true_relres(g, xc)) <= 1e-6 * rc["true_relres"]
    assert rc["launches"] == 1


@pytest.mark.parametrize("n_side", [4, 64, 181])
def test_cluster_solve_sizes(monkeypatch, n_side):
    """Poisson systems of 17, 4,096 and 32,761 rows (the last near the cluster's limit of
    16 x 2,048 rows; with 17 rows most CTAs own none) against the oracle restatement: the same
    info, iterations within +-2 of its envelope over dot-product orders, x within 10x its
    spread."""
    from test_gpu_batch import envelope
    A = FB.gen_poisson2d(n_side) if n_side != 4 else FB.gen_poisson2d(17, 1)
    n = len(A[0]) - 1
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    b = FB.rand_normal(n, 5 + n_side)
    monkeypatch.setenv("FIIM_PERSIST", "cluster")
    S = FB.Solver(A, F, variant="pdfiim")
    assert S.mode() == 3
    x = np.zeros(n)
    r = S.solve(b, x, tol=1e-8, nmax=3000)
    S.close()
    xo, infoo, lo, hi, spread = envelope("pdfiim", A, b, F, 3000)
    print(f"n={n}: cluster {r['iter']} iterations, oracle envelope [{lo},{hi}]")
    assert r["info"] == infoo == 0 and lo - 2 <= r["iter"] <= hi + 2
    assert np.linalg.norm(x - xo) <= (10 * spread + 1e-9) * np.linalg.norm(xo)


@pytest.mark.parametrize("nmax", [0, 1, 2, 5])
def test_cluster_solve_stops_at_nmax(golden, monkeypatch, nmax):
    """NMAX 0, 1, 2 and 5 end the cluster solve as they end the graph solve (info 3, the same
    iteration count and the same x to rounding)."""
    g = golden("poisson128_afiim")
    F = {k: g[k] for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    A = (g["Ai"], g["Aj"], g["Av"])
    res = {}
    for mode in ("cluster", "0"):
        monkeypatch.setenv("FIIM_PERSIST", mode)
        S = FB.Solver(A, F, variant="afiim")
        x = np.zeros(len(g["b"]))
        res[mode] = (S.solve(g["b"], x, tol=1e-8, nmax=nmax), x)
        S.close()
    (rc, xc), (rg, xg) = res["cluster"], res["0"]
    assert (rc["iter"], rc["info"]) == (rg["iter"], rg["info"]) and rc["info"] == 3
    assert np.linalg.norm(xc - xg) <= 1e-12 * max(np.linalg.norm(xg), 1e-300)
