"""Host-side logic (CPU only): generators, the host PDFIIM construction, the C-ABI surface.

No GPU compute is called here; on a machine without a B200 the GPU entry points must
fail loudly with FIIM_ENODEV instead of computing anything on the CPU.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import fiim_b200 as FB
import pyoracle as O
from conftest import ROOT, sub
import scipy.sparse as sp

HEADER = os.path.join(ROOT, "include", "fiim_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fiim_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = FB.lib()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/fiim_b200.h but not exported"
    assert sorted(FB.EXPORTS) == names


def test_reference_signature_overloads_exported():
    """The C++ drop-ins carry the reference's mangled names (AFIIM/ACIFIM/PDFIIM bicgstab.hpp)."""
    out = subprocess.run(["nm", "-D", "--defined-only", FB.LIB_PATH], capture_output=True, text=True).stdout
    syms = subprocess.run(["c++filt"], input=out, capture_output=True, text=True).stdout
    assert "EPBiCGSTAB(int, double*, int*, int*, double*, double, int, double*, int*, int*, double*, " \
           "double*, int*, int*, double*, double*, int*, int, int*)" in syms
    assert "PBiCGSTAB(int, double*, int*, int*, double*, double, int, double*, int*, int*, double*, double*, " \
           "int*, int*, double*, int*, int*, double*, int*, int*, int, char, double*, double*, int*, int, int*)" in syms
    assert "EPBiCGSTAB(sparseMatrix<int, int, double>&, std::vector<double, std::allocator<double> >&, double, " \
           "int, sparseMatrix<int, int, double>&, std::vector<double, std::allocator<double> >&, " \
           "sparseMatrix<int, int, double>&, std::vector<double, std::allocator<double> >&, double*, int*, int, " \
           "int*)" in syms


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_no_gpu_fails_loudly():
    A = FB.gen_poisson2d(8)
    F = {"Gi": A[0], "Gj": A[1], "Gv": A[2], "IDv": np.ones(64), "Hi": A[0], "Hj": A[1], "Hv": A[2]}
    with pytest.raises(FB.FiimError) as e:
        FB.Solver(A, F)
    assert e.value.rc == FB.FIIM_ENODEV
    x = np.zeros(64)
    with pytest.raises(FB.FiimError):
        FB.EPBiCGSTAB(64, A[2], A[1], A[0], np.ones(64), 1e-8, 10, A[2], A[1], A[0], np.ones(64), A[2], A[1],
                      A[0], x)
    assert not x.any()
    # the GPU factor construction and the row-partitioned solve
    with pytest.raises(FB.FiimError) as e:
        FB.pdfiim_build(A, 0.05, gpu=True)
    assert e.value.rc == FB.FIIM_ENODEV
    Fh = FB.pdfiim_build(A, 0.05)
    with pytest.raises(FB.FiimError) as e:
        FB.dist_emulate(A, Fh, np.ones(64), x, 2)
    assert e.value.rc == FB.FIIM_ENODEV
    rs = FB.dist_partition(A, Fh, 1)
    Al, Fl = FB.dist_local(A, Fh, rs, 0)
    with pytest.raises(FB.FiimError) as e:
        FB.DistSolver(0, 1, bytes(128), rs, Al, Fl)
    assert e.value.rc == FB.FIIM_ENODEV
    assert not x.any()


C_PROGRAM = r'''
#include <stdio.h>
#include <stdlib.h>
#include "fiim_b200.h"
int main(void) {
    fiim_options o;
    fiim_options_default(&o);
    if (o.variant != FIIM_AFIIM || o.precision != FIIM_FP64 || o.mode != 'E') return 1;
    if (o.reliable != 0.01 || o.max_refine != 50 || o.verified != 0) return 1;
    long nnz = fiim_gen_poisson2d(8, 8, NULL, NULL, NULL);
    int *Ai = malloc(sizeof(int) * 65), *Aj = malloc(sizeof(int) * nnz);
    double *Av = malloc(sizeof(double) * nnz);
    fiim_gen_poisson2d(8, 8, Ai, Aj, Av);
    int ng = 0, nh = 0;
    if (fiim_pdfiim_build(64, Ai, Aj, Av, 2, 2, 1, 0.05, -1, 'I', 'B', &ng, &nh, NULL, NULL, NULL, NULL, NULL,
                          NULL, NULL) != FIIM_OK) return 2;
    int *Gi = malloc(sizeof(int) * 65), *Gj = malloc(sizeof(int) * ng), *Hi = malloc(sizeof(int) * 65),
        *Hj = malloc(sizeof(int) * nh);
    double *Gv = malloc(sizeof(double) * ng), *Hv = malloc(sizeof(double) * nh), *D = malloc(sizeof(double) * 64);
    if (fiim_pdfiim_build(64, Ai, Aj, Av, 2, 2, 1, 0.05, -1, 'I', 'B', &ng, &nh, Gv, Gj, Gi, D, Hv, Hj, Hi) != FIIM_OK)
        return 3;
    if (Gi[64] != ng || Hi[64] != nh) return 4;
    fiim_solver_t h;
    int rc = fiim_solver_create(&h, 0, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                                NULL, NULL, NULL, NULL, &o);
    if (rc != FIIM_EARG || fiim_last_error()[0] == 0) return 5;
    printf("%d %d %d\n", (int)nnz, ng, nh);
    return 0;
}
'''


def test_c_program_builds_and_calls_the_library(tmp_path):
    """A C99 program includes include/fiim_b200.h, links libfiim_b200.so and calls host-side
    entry points (options, a generator, the two-call PDFIIM construction, argument errors)."""
    src = tmp_path / "t.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "t"
    pkg = os.path.dirname(FB.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-L", pkg,
                    "-lfiim_b200", f"-Wl,-rpath,{pkg}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out
    nnz, ng, nh = (int(v) for v in out.stdout.split())
    A = FB.gen_poisson2d(8)
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1)
    assert nnz == len(A[1]) and ng == len(F["Gj"]) and nh == len(F["Hj"])


def test_options_layout_matches_the_header():
    """The ctypes mirror of fiim_options reads the C defaults field for field."""
    o = FB.Options()
    FB.lib().fiim_options_default(C.byref(o))
    assert (o.variant, o.precision, o.memory, o.mode, o.nr) == (FB._VARIANTS["afiim"], FB.FP64, FB.MEM_HOST, b"E", 1)
    assert (o.inner_tol, o.inner_nmax, o.max_refine) == (1e-5, 1000, 50)
    assert (o.verified, o.max_restarts, o.reliable) == (0, 4, 0.01)


def test_bad_arguments_rejected_before_device():
    lib = FB.lib()
    h = C.c_void_p(0)
    assert lib.fiim_solver_create(C.byref(h), 0, None, None, None, None, None, None, None, None, None, None,
                                  None, None, None, None, None, None, None) == FB.FIIM_EARG
    assert "n <= 0" in lib.fiim_last_error().decode()
    x = np.zeros(4)
    r = FB.Result()
    assert lib.fiim_solver_solve(None, x.ctypes, x.ctypes, C.c_double(1e-8), 10, C.byref(r)) == FB.FIIM_EARG
    # ACIFIM modes 'I' and 'J' are triangular solves, not the factored inverse
    A = FB.gen_poisson2d(2)
    rc = lib.fiim_PBiCGSTAB_acifim(4, *[a.ctypes for a in (A[2], A[1], A[0])], x.ctypes, C.c_double(1e-8), 5,
                                   *[a.ctypes for a in (A[2], A[1], A[0], x, A[2], A[1], A[0])],
                                   *[a.ctypes for a in (A[2], A[1], A[0], A[2], A[1], A[0])], 1, C.c_char(b"I"),
                                   x.ctypes, C.byref(C.c_double()), C.byref(C.c_int()), 0, C.byref(C.c_int()))
    assert rc == FB.FIIM_EARG


# ----------------------------------------------------------------------------- generators
def test_poisson2d():
    Ai, Aj, Av = FB.gen_poisson2d(128)
    n = 128 * 128
    assert len(Ai) == n + 1 and Ai[-1] == 81408
    assert np.all(np.diff(Ai) >= 3)
    for i in (0, 77, n - 1):
        cols = Aj[Ai[i]:Ai[i + 1]]
        assert np.all(np.diff(cols) > 0)
        assert Av[Ai[i] + list(cols).index(i)] == 4.0
    assert FB.model_rhs((Ai, Aj, Av))[200] == 0.0      # interior row sum


def test_convdiff3d_structure():
    N = 12
    Ai, Aj, Av = FB.gen_convdiff3d(N, 0.5)
    n = N ** 3
    assert Ai[-1] == 7 * n - 6 * N * N
    rows = np.repeat(np.arange(n), np.diff(Ai))
    assert np.all(np.diff(Aj)[np.diff(rows) == 0] > 0)               # ascending columns
    assert np.all(Av[Aj == rows] == 7.5)
    assert np.all(Av[Aj < rows] == -1.5) and np.all(Av[Aj > rows] == -1.0)
    interior = N * N * (N // 2) + N * (N // 2) + N // 2
    assert abs(Av[Ai[interior]:Ai[interior + 1]].sum()) < 1e-15
    # the 128^3 workload's size without building it
    assert FB.lib().fiim_gen_convdiff3d(128, C.c_double(0.5), None, None, None) == 14581760


def test_convdiff2d_and_batch_params():
    sides = []
    for k in range(256):
        side, diff, theta, pe = FB.batch_params(20261203, k)
        assert 32 <= side <= 256 and 0.1 <= diff <= 10 and 0 <= theta < 6.2832 and 0 < pe <= 1
        sides.append(side)
    assert FB.batch_params(20261203, 5) == FB.batch_params(20261203, 5)
    assert 100 < np.mean(sides) < 190
    side, diff, theta, pe = FB.batch_params(20261203, 3)
    Ai, Aj, Av = FB.gen_convdiff2d(20, diff, theta, pe)
    assert Ai[-1] == 5 * 400 - 80
    rows = np.repeat(np.arange(400), np.diff(Ai))
    off = Av[Aj != rows]
    assert np.all(off < 0)                                           # M-matrix sign pattern
    s = np.zeros(400)
    np.add.at(s, rows, Av)
    assert np.all(s > -1e-12)                                        # weak diagonal dominance


def test_zipf_rows():
    n = 20000
    scale = FB.zipf_scale(n, sample=n)
    Ai, Aj, Av = FB.gen_zipf(n, scale)
    lens = np.diff(Ai)
    assert abs(lens.mean() - 16) < 0.25 and lens.min() >= 1 and lens.max() <= 512
    rows = np.repeat(np.arange(n), lens)
    d = Av[Aj == rows]
    assert len(d) == n
    off = np.zeros(n)
    np.add.at(off, rows[Aj != rows], np.abs(Av[Aj != rows]))
    nz = off > 0
    assert np.allclose(d[nz], 1.1 * off[nz])
    assert np.all(np.diff(Aj)[np.diff(rows) == 0] > 0)


def test_rand_normal():
    x = FB.rand_normal(200000, 7)
    assert abs(x.mean()) < 0.01 and abs(x.std() - 1) < 0.01
    assert np.array_equal(x[:10], FB.rand_normal(10, 7))


# ----------------------------------------------------------------------------- construction
def test_host_pdfiim_matches_golden_factors(golden):
    g = golden("convdiff16_pdfiim")
    F = FB.pdfiim_build((g["Ai"], g["Aj"], g["Av"]), 0.05, 2, 2, 1, -1, "I", "B")
    for k in ("Gi", "Gj", "Gv", "Hi", "Hj", "Hv", "IDv"):
        assert np.array_equal(F[k], g[k]), k


def test_host_pdfiim_matches_golden_sherman2(golden):
    g = golden("sherman2")
    F = FB.pdfiim_build((g["Ai"], g["Aj"], g["Av"]), 0.01, 2, 2, 1, -1, "I", "B")
    for k in ("Gi", "Gj", "Gv", "Hi", "Hj", "Hv", "IDv"):
        assert np.array_equal(F[k], g["pdfiim_" + k]), k


@pytest.mark.skipif(not O.have_ref("pdfiim"), reason="oracle/_ref not built")
@pytest.mark.parametrize("params", [(1, 1, 1, -1, "I"), (3, 2, 2, -1, "1"), (2, 3, 2, 9, "2"), (2, 2, 1, 5, "I")])
def test_host_pdfiim_matches_live_reference(params):
    pf, lf, po, ws, ft = params
    rng = np.random.default_rng(pf * 7 + lf)
    A = FB.gen_convdiff2d(30, float(rng.uniform(0.2, 4)), float(rng.uniform(0, 6.2)), 0.9)
    R = O.pdfiim_build(A, 0.05, pf, lf, po, ws, ft, "B")
    M = FB.pdfiim_build(A, 0.05, pf, lf, po, ws, ft, "B")
    for k in ("Gi", "Gj", "Gv", "Hi", "Hj", "Hv", "IDv"):
        assert np.array_equal(R[k], M[k]), k


def test_host_pdfiim_rejects_unserved_patterns():
    A = FB.gen_poisson2d(4)
    for patt in "LU":
        with pytest.raises(FB.FiimError):
            FB.pdfiim_build(A, 0.05, patt=patt)


def test_block_diag_matches_scipy():
    """The batched handle's concatenation: block-diagonal CSR in global numbering, with the
    systems' first rows."""
    import scipy.sparse as sp
    mats = [FB.gen_convdiff2d(s, 1.0 + s, 0.7, 0.5) for s in (3, 5, 4)]
    (Ai, Aj, Av), rows = FB.block_diag(mats)
    ref = sp.block_diag([sp.csr_matrix((m[2], m[1], m[0])) for m in mats], format="csr")
    assert np.array_equal(Ai, ref.indptr) and np.array_equal(Aj, ref.indices) and np.array_equal(Av, ref.data)
    assert list(rows) == [0, 9, 34, 50]
    assert Ai.dtype == np.int32 and Aj.dtype == np.int32


def test_handles_close_on_leaving_a_with_block():
    """Solver, DistSolver, BatchSolver and BlockSolver are context managers whose exit calls
    close(), also when the block raises."""
    for cls in (FB.Solver, FB.DistSolver, FB.BatchSolver, FB.BlockSolver):
        assert issubclass(cls, FB._Handle)

    class Probe(FB._Handle):
        closed = 0

        def close(self):
            Probe.closed += 1

    with Probe() as h:
        assert isinstance(h, Probe)
    with pytest.raises(ValueError):
        with Probe():
            raise ValueError("inside")
    assert Probe.closed == 2


ACIFIM_KEYS = ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv", "Li", "Lj", "Lv", "Ui", "Uj", "Uv")


def _same_factors(F, R):
    for k in ACIFIM_KEYS:
        assert F[k].dtype == np.asarray(R[k]).dtype and np.array_equal(F[k], R[k]), k


@pytest.mark.parametrize("name,prefix,dtols", [("convdiff2d48_acifim", "", (0.1, 0.05)),
                                               ("sherman2", "acifim_", (0.01, 0.01))])
def test_host_acifim_matches_golden_factors(golden, name, prefix, dtols):
    """The library's ACIFIM construction against the factors the reference built for the
    committed fixtures (ACIFIM/src/prec.cpp:127-1052), all five factors bit for bit."""
    g = golden(name)
    F = FB.acifim_build((g["Ai"], g["Aj"], g["Av"]), *dtols, with_lu=True)
    _same_factors(F, sub(g, prefix))


def _random_system(n, seed, zero_diag=0):
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for i in range(n):
        k = int(rng.integers(1, 9))
        c = rng.choice(n, k, replace=False)
        rows.append(np.full(k + 1, i))
        cols.append(np.concatenate([c, [i]]))
    M = sp.csr_matrix((rng.uniform(-1, 1, sum(len(c) for c in cols)), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    M.sum_duplicates()
    M = M + sp.diags(np.abs(M).sum(axis=1).A1 * 1.2)
    M = M.tocsr()
    M.sort_indices()
    if zero_diag:
        for i in rng.choice(n, zero_diag, replace=False):
            M[i, i] = 0.0
    M.sort_indices()
    return M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data.copy()


@pytest.mark.skipif(not O.have_ref("acifim"), reason="oracle/_ref not built")
@pytest.mark.parametrize("case", [
    dict(system="convdiff", k=3, dtols=(0.1, 0.05)),
    dict(system="convdiff", k=6, dtols=(0.1, 0.05)),
    dict(system="convdiff", k=9, dtols=(0.02, 0.01), element_limit=4, filtit=6, coeff=1.5),
    dict(system="random", seed=1, dtols=(0.1, 0.05)),
    dict(system="random", seed=2, dtols=(0.01, 0.005), element_limit=3, filtit=30, coeff=2.0),
    dict(system="random", seed=3, dtols=(0.05, 0.05), shift=0.2, eta=0.5),
    dict(system="random", seed=4, dtols=(0.1, 0.05), zero_diag=40),
    dict(system="single", dtols=(0.1, 0.05)),
])
def test_host_acifim_matches_live_reference(case):
    """Against the reference's own acifim, compiled here, on 2D convection-diffusion systems of
    the batched benchmark's family, random nonsymmetric systems (repeated filter passes with
    a small element limit, shift and eta, rows whose diagonal is zero) and a 1 x 1 system."""
    case = dict(case)
    system, dtols = case.pop("system"), case.pop("dtols")
    if system == "convdiff":
        side, diff, theta, pe = FB.batch_params(20261203, case.pop("k"))
        A = FB.gen_convdiff2d(side, diff, theta, pe)
    elif system == "random":
        A = _random_system(3000, case.pop("seed"), case.pop("zero_diag", 0))
    else:
        A = (np.array([0, 1], np.int32), np.array([0], np.int32), np.array([2.5]))
    R, cerr = O.acifim_build(A, *dtols, **case)
    assert cerr == 0
    _same_factors(FB.acifim_build(A, *dtols, with_lu=True, **case), R)


def test_host_acifim_threads_build_independent_systems():
    """Each thread keeps its own result between the sizing and copy-out calls, so systems
    built on a thread pool come out as built one by one."""
    from concurrent.futures import ThreadPoolExecutor
    systems = [FB.gen_convdiff2d(*[FB.batch_params(7, k)[0]] + list(FB.batch_params(7, k)[1:])) for k in range(12)]
    one = [FB.acifim_build(A, 0.1, 0.05) for A in systems]
    with ThreadPoolExecutor(6) as ex:
        par = list(ex.map(lambda A: FB.acifim_build(A, 0.1, 0.05), systems))
    for F, R in zip(par, one):
        assert all(np.array_equal(F[k], R[k]) for k in R)


def test_host_acifim_nan_pivot_fails():
    """A NaN in A reaches a Schur complement: the reference's acifim returns 1 there, the
    library returns FIIM_EARG."""
    A = FB.gen_convdiff2d(8, 1.0, 0.3, 0.5)
    Av = A[2].copy()
    Av[5] = np.nan
    with pytest.raises(FB.FiimError):
        FB.acifim_build((A[0], A[1], Av), 0.1, 0.05)
    if O.have_ref("acifim"):
        assert O.acifim_build((A[0], A[1], Av), 0.1, 0.05)[1] == 1


@pytest.mark.parametrize("name,prefix,dtol", [("sherman2", "afiim9e-6_", 9e-6), ("sherman2", "afiim0.1_", 0.1),
                                              ("poisson128_afiim", "", 0.1)])
def test_host_afiim_matches_golden_factors(golden, name, prefix, dtol):
    """The library's AFIIM construction against the factors the reference built for the
    committed fixtures (AFIIM/src/prec.cpp:101-767), bit for bit."""
    g = golden(name)
    F = FB.afiim_build((g["Ai"], g["Aj"], g["Av"]), dtol)
    R = sub(g, prefix)
    for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv"):
        assert F[k].dtype == R[k].dtype and np.array_equal(F[k], R[k]), k


@pytest.mark.skipif(not O.have_ref("afiim"), reason="oracle/_ref not built")
@pytest.mark.parametrize("case", [
    dict(system="zipf", n=20000, dtol=0.1),
    dict(system="random", seed=5, dtol=0.05),
    dict(system="random", seed=6, dtol=0.1, shift=0.1, eta=0.4),
    dict(system="random", seed=7, dtol=0.02, zero_diag=30),
    dict(system="convdiff", k=4, dtol=0.1),
])
def test_host_afiim_matches_live_reference(case):
    """Against the reference's own afiim, compiled here: the multi-RHS benchmark's Zipf family,
    random nonsymmetric systems (shift and eta, rows whose diagonal is zero), and a 2D
    convection-diffusion system."""
    case = dict(case)
    system, dtol = case.pop("system"), case.pop("dtol")
    if system == "zipf":
        n = case.pop("n")
        A = FB.gen_zipf(n, FB.zipf_scale(4000000, sample=200000))
    elif system == "random":
        A = _random_system(3000, case.pop("seed"), case.pop("zero_diag", 0))
    else:
        side, diff, theta, pe = FB.batch_params(20261203, case.pop("k"))
        A = FB.gen_convdiff2d(side, diff, theta, pe)
    R = O.afiim_build(A, dtol, **case)
    F = FB.afiim_build(A, dtol, **case)
    for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv"):
        assert F[k].dtype == R[k].dtype and np.array_equal(F[k], R[k]), k
