"""ORACLE TEST INFRASTRUCTURE — not product code.

ctypes bindings for the two checkers under oracle/:
  * liboracle.so          — plain-C restatement of the solve phase (fiim_oracle.c)
  * _ref/libref_<pkg>.so  — the reference's own sources compiled against the MKL shim
Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
module, and only to check or to time the reference's CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# The reference tree: FIIM_REFERENCE, else a checkout named `reference` beside this repository.
REFERENCE = os.environ.get("FIIM_REFERENCE",
                           os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

_libs: dict[str, C.CDLL] = {}


def build(ref: bool = True) -> None:
    """Compile the restatement (always) and, when the reference tree exists, oracle/_ref."""
    targets = ["restatement"]
    if ref and os.path.isdir(REFERENCE):
        targets += ["ref", "REF=" + REFERENCE]
    subprocess.run(["make", "-s", "-C", HERE, *targets], check=True)


def have_ref(pkg: str = "afiim") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{pkg}.so"))


def _lib(name: str) -> C.CDLL:
    if name in _libs:
        return _libs[name]
    path = os.path.join(HERE, "liboracle.so") if name == "oracle" else os.path.join(REF_DIR, f"libref_{name}.so")
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C {HERE}`")
    lib = C.CDLL(path, mode=os.RTLD_LOCAL)
    _libs[name] = lib
    return lib


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ----------------------------------------------------------------------------- restatement
ORC_AFIIM, ORC_PDFIIM, ORC_ACIFIM = 0, 1, 2
ORC_GENERAL, ORC_UPPER, ORC_LOWER = 0, 1, 2
_VARIANT = {"afiim": ORC_AFIIM, "pdfiim": ORC_PDFIIM, "acifim": ORC_ACIFIM}


def csr_mv(Ai, Aj, Av, x, fill=ORC_GENERAL):
    lib = _lib("oracle")
    n = len(Ai) - 1
    y = np.zeros(n)
    lib.orc_csr_mv(C.c_int(n), _i(Ai).ctypes, _i(Aj).ctypes, _d(Av).ctypes, C.c_int(fill),
                   _d(x).ctypes, y.ctypes)
    return y


def csr_mv_trans(Ai, Aj, Av, x, fill=ORC_GENERAL):
    lib = _lib("oracle")
    n = len(Ai) - 1
    y = np.zeros(n)
    lib.orc_csr_mv_trans(C.c_int(n), _i(Ai).ctypes, _i(Aj).ctypes, _d(Av).ctypes, C.c_int(fill),
                         _d(x).ctypes, y.ctypes)
    return y


def csr_mv_sym_upper(Ai, Aj, Av, x):
    lib = _lib("oracle")
    n = len(Ai) - 1
    y = np.zeros(n)
    lib.orc_csr_mv_sym_upper(C.c_int(n), _i(Ai).ctypes, _i(Aj).ctypes, _d(Av).ctypes,
                             _d(x).ctypes, y.ctypes)
    return y


def prec_apply(F, r, sym=False):
    """z = G * (IDv o (H * r)) (or G * (IDv o (G^T r)) when sym)."""
    lib = _lib("oracle")
    n = len(F["IDv"])
    out, tm = np.zeros(n), np.zeros(n)
    if sym:
        lib.orc_prec_apply_sym(C.c_int(n), _i(F["Gi"]).ctypes, _i(F["Gj"]).ctypes, _d(F["Gv"]).ctypes,
                               _d(F["IDv"]).ctypes, _d(r).ctypes, out.ctypes, tm.ctypes)
    else:
        lib.orc_prec_apply(C.c_int(n), _i(F["Gi"]).ctypes, _i(F["Gj"]).ctypes, _d(F["Gv"]).ctypes,
                           _d(F["IDv"]).ctypes, _i(F["Hi"]).ctypes, _i(F["Hj"]).ctypes,
                           _d(F["Hv"]).ctypes, _d(r).ctypes, out.ctypes, tm.ctypes)
    return out


def prec_apply_combined(F, r, nr):
    lib = _lib("oracle")
    n = len(F["IDv"])
    out, work = np.zeros(n), np.zeros(3 * n)
    a = [_i(F[k]) if k[1] in "ij" else _d(F[k]) for k in
         ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv", "Li", "Lj", "Lv", "Ui", "Uj", "Uv")]
    lib.orc_prec_apply_combined(C.c_int(n), C.c_int(nr), *[x.ctypes for x in a], _d(r).ctypes,
                                out.ctypes, work.ctypes)
    return out


def set_dot_blocks(blocks: int) -> None:
    """Sum dots and norms over `blocks` contiguous blocks, as the shim does on that many threads."""
    _lib("oracle").orc_set_dot_blocks(C.c_int(blocks))


def bicgstab(variant, A, b, F, tol=1e-8, nmax=500, x0=None, issym=False, mode="E", nr=1):
    """Restated EPBiCGSTAB / PBiCGSTAB. Returns (x, resval, iter, info)."""
    lib = _lib("oracle")
    Ai, Aj, Av = _i(A[0]), _i(A[1]), _d(A[2])
    n = len(Ai) - 1
    x = np.zeros(n) if x0 is None else _d(x0).copy()
    resval, it, info = C.c_double(0), C.c_int(0), C.c_int(-1)
    empty_i, empty_d = np.zeros(1, np.int32), np.zeros(1)

    def g(k, dflt):
        return F[k] if (k in F and F[k] is not None) else dflt

    Hi, Hj, Hv = _i(g("Hi", empty_i)), _i(g("Hj", empty_i)), _d(g("Hv", empty_d))
    Li, Lj, Lv = _i(g("Li", empty_i)), _i(g("Lj", empty_i)), _d(g("Lv", empty_d))
    Ui, Uj, Uv = _i(g("Ui", empty_i)), _i(g("Uj", empty_i)), _d(g("Uv", empty_d))
    rc = lib.orc_bicgstab(
        C.c_int(_VARIANT[variant]), C.c_int(int(issym)), C.c_char(mode.encode()), C.c_int(nr),
        C.c_int(n), Ai.ctypes, Aj.ctypes, Av.ctypes, _d(b).ctypes, C.c_double(tol), C.c_int(nmax),
        _i(F["Gi"]).ctypes, _i(F["Gj"]).ctypes, _d(F["Gv"]).ctypes, _d(F["IDv"]).ctypes,
        Hi.ctypes, Hj.ctypes, Hv.ctypes, Li.ctypes, Lj.ctypes, Lv.ctypes, Ui.ctypes, Uj.ctypes,
        Uv.ctypes, x.ctypes, C.byref(resval), C.byref(it), C.byref(info))
    if rc != 0:
        raise ValueError("orc_bicgstab rejected its arguments")
    return x, resval.value, it.value, info.value


# ----------------------------------------------------------------------------- reference
def set_threads(t: int, pkg: str = "afiim") -> None:
    _lib(pkg).ref_set_threads(C.c_int(t))


def _collect(lib, h, with_lu=False):
    sizes = np.zeros(5, dtype=np.int64)
    lib.ref_factors_sizes(C.c_void_p(h), sizes.ctypes)
    n, ng, nh, nl, nu = (int(s) for s in sizes)
    F = {"Gv": np.zeros(ng), "Gj": np.zeros(ng, np.int32), "Gi": np.zeros(n + 1, np.int32),
         "IDv": np.zeros(n), "Hv": np.zeros(nh), "Hj": np.zeros(nh, np.int32),
         "Hi": np.zeros(n + 1, np.int32)}
    if with_lu:
        F.update({"Lv": np.zeros(nl), "Lj": np.zeros(nl, np.int32), "Li": np.zeros(n + 1, np.int32),
                  "Uv": np.zeros(nu), "Uj": np.zeros(nu, np.int32), "Ui": np.zeros(n + 1, np.int32)})
    else:
        F.update({k: None for k in ("Lv", "Lj", "Li", "Uv", "Uj", "Ui")})
    if nh == 0 and not with_lu:
        F["Hv"] = F["Hj"] = F["Hi"] = None
    ptr = lambda k: (F[k].ctypes if F.get(k) is not None else None)
    lib.ref_factors_get(C.c_void_p(h), *[ptr(k) for k in
                        ("Gv", "Gj", "Gi", "IDv", "Hv", "Hj", "Hi", "Lv", "Lj", "Li", "Uv", "Uj", "Ui")])
    lib.ref_factors_free(C.c_void_p(h))
    return F


def read_matrix(path: str):
    """Reference Matrix Market reader (AFIIM/src/rw_matrix.cpp:62-216) -> (Ai, Aj, Av)."""
    lib = _lib("afiim")
    lib.ref_read_matrix.restype = C.c_void_p
    n, nnz = C.c_int(0), C.c_int(0)
    h = lib.ref_read_matrix(path.encode(), C.byref(n), C.byref(nnz))
    Av, Aj, Ai = np.zeros(nnz.value), np.zeros(nnz.value, np.int32), np.zeros(n.value + 1, np.int32)
    lib.ref_csr_get(C.c_void_p(h), Av.ctypes, Aj.ctypes, Ai.ctypes)
    lib.ref_free_csr(C.c_void_p(h))
    return Ai, Aj, Av


def read_rhs(path: str, n: int):
    lib = _lib("afiim")
    out = np.zeros(n)
    m = lib.ref_read_rhs(path.encode(), out.ctypes, C.c_int(n))
    assert m == n, (m, n)
    return out


def afiim_build(A, dtol, elem_per_rowcol=10, growth=5, eta=0.0, shift=0.0):
    """Reference afiim (AFIIM/src/prec.cpp:101-767); driver defaults AFIIM/example/example.cpp:37-39."""
    lib = _lib("afiim")
    lib.ref_afiim_build.restype = C.c_void_p
    Ai, Aj, Av = _i(A[0]), _i(A[1]), _d(A[2])
    h = lib.ref_afiim_build(C.c_int(len(Ai) - 1), Av.ctypes, Aj.ctypes, Ai.ctypes, C.c_double(dtol),
                            C.c_int(elem_per_rowcol), C.c_int(growth), C.c_double(eta), C.c_double(shift))
    return _collect(lib, h)


def pdfiim_build(A, ftol, prefill=1, lfill=1, postfill=1, warpsize=-1, filttype="I", patt="B"):
    """Reference pdfiim (PDFIIM/src/parPrec.cpp:95-588); the example passes 'I','B' (pdfiim.cpp:95-104)."""
    lib = _lib("pdfiim")
    lib.ref_pdfiim_build.restype = C.c_void_p
    Ai, Aj, Av = _i(A[0]), _i(A[1]), _d(A[2])
    h = lib.ref_pdfiim_build(C.c_int(len(Ai) - 1), Av.ctypes, Aj.ctypes, Ai.ctypes, C.c_int(prefill),
                             C.c_int(lfill), C.c_int(postfill), C.c_double(ftol), C.c_int(warpsize),
                             C.c_char(filttype.encode()), C.c_char(patt.encode()))
    return _collect(lib, h)


def acifim_build(A, dtol1, dtol2, elem_per_rowcol=30, growth=5, eta=0.0, shift=0.0, coeff=2.0,
                 element_limit=200, filtit=30):
    """Reference acifim (ACIFIM/src/prec.cpp:127-1052); driver defaults ACIFIM/example/example.cpp:42-47.
    Returns (factors or None, construction status)."""
    lib = _lib("acifim")
    lib.ref_acifim_build.restype = C.c_void_p
    Ai, Aj, Av = _i(A[0]), _i(A[1]), _d(A[2])
    cerr = C.c_int(0)
    h = lib.ref_acifim_build(C.c_int(len(Ai) - 1), Av.ctypes, Aj.ctypes, Ai.ctypes, C.c_double(dtol1),
                             C.c_double(dtol2), C.c_int(elem_per_rowcol), C.c_int(growth),
                             C.c_double(eta), C.c_double(shift), C.c_double(coeff),
                             C.c_int(element_limit), C.c_int(filtit), C.byref(cerr))
    if not h:
        return None, cerr.value
    return _collect(lib, h, with_lu=True), cerr.value


def ref_solve(variant, A, b, F, tol=1e-8, nmax=500, x0=None, issym=False, mode="E", nr=1, verbose=0):
    """The reference's own EPBiCGSTAB / PBiCGSTAB. Returns (x, resval, iter, info)."""
    Ai, Aj, Av = _i(A[0]), _i(A[1]), _d(A[2])
    n = len(Ai) - 1
    x = np.zeros(n) if x0 is None else _d(x0).copy()
    b = _d(b).copy()
    resval, it, info = C.c_double(0), C.c_int(0), C.c_int(-1)
    G = [_i(F["Gj"]), _i(F["Gi"])]
    Gv, IDv = _d(F["Gv"]), _d(F["IDv"])
    if variant == "afiim":
        lib = _lib("afiim")
        lib.ref_afiim_solve(C.c_int(n), Av.ctypes, Aj.ctypes, Ai.ctypes, b.ctypes, C.c_double(tol),
                            C.c_int(nmax), Gv.ctypes, G[0].ctypes, G[1].ctypes, IDv.ctypes,
                            _d(F["Hv"]).ctypes, _i(F["Hj"]).ctypes, _i(F["Hi"]).ctypes, x.ctypes,
                            C.byref(resval), C.byref(it), C.c_int(verbose), C.byref(info))
    elif variant == "pdfiim":
        lib = _lib("pdfiim")
        if issym:
            Hv, Hj, Hi = np.zeros(1), np.zeros(1, np.int32), np.zeros(1, np.int32)
        else:
            Hv, Hj, Hi = _d(F["Hv"]), _i(F["Hj"]), _i(F["Hi"])
        lib.ref_pdfiim_solve(C.c_int(n), C.c_int(int(issym)), Av.ctypes, Aj.ctypes, Ai.ctypes, b.ctypes,
                             C.c_double(tol), C.c_int(nmax), Gv.ctypes, G[0].ctypes, G[1].ctypes,
                             IDv.ctypes, Hv.ctypes, Hj.ctypes, Hi.ctypes, x.ctypes, C.byref(resval),
                             C.byref(it), C.c_int(verbose), C.byref(info))
    elif variant == "acifim":
        lib = _lib("acifim")
        lu = [_d(F["Lv"]), _i(F["Lj"]), _i(F["Li"]), _d(F["Uv"]), _i(F["Uj"]), _i(F["Ui"])]
        lib.ref_acifim_solve(C.c_int(n), Av.ctypes, Aj.ctypes, Ai.ctypes, b.ctypes, C.c_double(tol),
                             C.c_int(nmax), Gv.ctypes, G[0].ctypes, G[1].ctypes, IDv.ctypes,
                             _d(F["Hv"]).ctypes, _i(F["Hj"]).ctypes, _i(F["Hi"]).ctypes,
                             *[a.ctypes for a in lu], C.c_int(nr), C.c_char(mode.encode()), x.ctypes,
                             C.byref(resval), C.byref(it), C.c_int(verbose), C.byref(info))
    else:
        raise ValueError(variant)
    return x, resval.value, it.value, info.value


class RefPdfiimSystem:
    """The reference's PDFIIM system held as its own sparseMatrix objects and std::vectors
    (built once), so that each run() times the reference's EPBiCGSTAB call by itself
    (PDFIIM/src/bicgstab.cpp:80-310), without marshalling the arrays into it."""

    def __init__(self, A, F, issym=False):
        lib = _lib("pdfiim")
        lib.ref_pdfiim_prepare.restype = C.c_void_p
        lib.ref_pdfiim_run.restype = C.c_double
        self._lib = lib
        self._keep = [_d(A[2]), _i(A[1]), _i(A[0]), _d(F["Gv"]), _i(F["Gj"]), _i(F["Gi"]), _d(F["IDv"])]
        if issym:
            self._keep += [np.zeros(1), np.zeros(1, np.int32), np.zeros(1, np.int32)]
        else:
            self._keep += [_d(F["Hv"]), _i(F["Hj"]), _i(F["Hi"])]
        self.n = len(self._keep[2]) - 1
        self._h = lib.ref_pdfiim_prepare(C.c_int(self.n), C.c_int(int(issym)), *[a.ctypes for a in self._keep])

    def run(self, b, tol=1e-8, nmax=1200, x0=None):
        """One EPBiCGSTAB call. Returns (x, resval, iter, info, seconds inside the call)."""
        x = np.zeros(self.n) if x0 is None else _d(x0).copy()
        resval, it, info = C.c_double(0), C.c_int(0), C.c_int(-1)
        secs = self._lib.ref_pdfiim_run(C.c_void_p(self._h), _d(b).ctypes, x.ctypes, C.c_double(tol),
                                        C.c_int(nmax), C.byref(resval), C.byref(it), C.byref(info))
        return x, resval.value, it.value, info.value, secs

    def close(self):
        if self._h:
            self._lib.ref_pdfiim_release(C.c_void_p(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
