"""Python mirror of the reference's solve-phase interface over libfiim_b200.so.

The functions keep the reference's names, argument meaning and in/out convention:

* ``EPBiCGSTAB``        — AFIIM/src/bicgstab.hpp:82-100 (pointer form)
* ``EPBiCGSTAB_pdfiim`` — PDFIIM/src/bicgstab.hpp:75-86 (sparseMatrix form, as CSR arrays)
* ``PBiCGSTAB``         — ACIFIM/src/bicgstab.hpp:94-120 (modes 'E' and 'C')

``x`` is the initial guess in and the solution out (updated in place); the scalars come
back as ``(resval, iter, info)`` with the reference's ``info`` codes (0 converged,
1 diverged, 2 stagnated, 3 NMAX). A GPU-side failure raises ``FiimError``; there is no
CPU fallback.

``Solver`` wraps the handle API (set up once, solve many times) for host (numpy) or
device (torch CUDA tensor) arrays, in FP64 or mixed precision; ``BatchSolver`` and
``BlockSolver`` wrap the batched uneven systems and the multi-RHS block solve;
``DistSolver`` is one rank of a solve split into row blocks over several GPUs
(``dist_emulate`` runs all blocks on one GPU). Generators, the PDFIIM construction (host or
GPU), the Matrix Market readers and the factor file are exposed for tests, benchmarks and
callers without the reference library.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfiim_b200.so")

FIIM_OK, FIIM_EARG, FIIM_ECUDA, FIIM_ENOMEM, FIIM_ENODEV, FIIM_ETIMEOUT = 0, -1, -2, -3, -4, -5
AFIIM, PDFIIM, ACIFIM = 0, 1, 2
FP64, MIXED_FP32, MIXED_BF16 = 0, 1, 2
MEM_HOST, MEM_DEVICE = 0, 1
_VARIANTS = {"afiim": AFIIM, "pdfiim": PDFIIM, "acifim": ACIFIM}
_PRECISIONS = {"fp64": FP64, "fp32": MIXED_FP32, "bf16": MIXED_BF16}

# Every extern "C" symbol include/fiim_b200.h declares.
EXPORTS = (
    "fiim_last_error", "fiim_dropin_cache", "fiim_options_default", "fiim_EPBiCGSTAB_afiim", "fiim_EPBiCGSTAB_pdfiim",
    "fiim_PBiCGSTAB_acifim", "fiim_solver_create", "fiim_solver_solve", "fiim_solver_device_bytes",
    "fiim_solver_spmv_shape", "fiim_solver_apply", "fiim_solver_kernel_times", "fiim_solver_kernel_times_seq", "fiim_solver_mode",
    "fiim_solver_set_wait_limit", "fiim_solver_test_stall", "fiim_solver_iteration_bytes", "fiim_solver_matrix_bytes",
    "fiim_solver_destroy", "fiim_batch_create", "fiim_batch_solve", "fiim_batch_destroy",
    "fiim_block_create", "fiim_block_solve", "fiim_block_apply", "fiim_block_spmm_shape", "fiim_block_destroy",
    "fiim_spmv", "fiim_prec_apply", "fiim_prec_apply_noalloc",
    "fiim_gen_poisson2d", "fiim_gen_convdiff3d", "fiim_gen_convdiff2d", "fiim_gen_batch_params",
    "fiim_gen_zipf", "fiim_gen_zipf_mean", "fiim_rand_normal", "fiim_model_rhs", "fiim_pdfiim_build", "fiim_pdfiim_build_gpu",
    "fiim_acifim_build", "fiim_afiim_build",
    "fiim_read_mtx", "fiim_read_rhs", "fiim_factors_save", "fiim_factors_load",
    "fiim_dist_unique_id", "fiim_dist_partition", "fiim_dist_plan", "fiim_dist_create", "fiim_dist_solve",
    "fiim_dist_destroy", "fiim_dist_emulate",
)


class FiimError(RuntimeError):
    def __init__(self, rc: int, msg: str):
        super().__init__(f"fiim_b200 error {rc}: {msg}")
        self.rc = rc


class Options(C.Structure):
    _fields_ = [("variant", C.c_int), ("issym", C.c_int), ("precision", C.c_int), ("memory", C.c_int),
                ("mode", C.c_char), ("nr", C.c_int), ("autotune", C.c_int), ("verbose", C.c_int),
                ("inner_tol", C.c_double), ("inner_nmax", C.c_int), ("max_refine", C.c_int),
                ("verified", C.c_int), ("max_restarts", C.c_int), ("reliable", C.c_double)]


class Result(C.Structure):
    _fields_ = [("resval", C.c_double), ("true_relres", C.c_double), ("iter", C.c_int), ("info", C.c_int),
                ("refine_steps", C.c_int), ("device_ms", C.c_double), ("launches", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib() -> C.CDLL:
    """Load libfiim_b200.so (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} not built; run `make -C {HERE}`")
        L = C.CDLL(LIB_PATH, mode=os.RTLD_LOCAL)
        L.fiim_last_error.restype = C.c_char_p
        L.fiim_solver_device_bytes.restype = C.c_int64
        for name in ("fiim_gen_poisson2d", "fiim_gen_convdiff3d", "fiim_gen_convdiff2d", "fiim_gen_zipf"):
            getattr(L, name).restype = C.c_long
        L.fiim_gen_zipf_mean.restype = C.c_double
        L.fiim_solver_iteration_bytes.restype = C.c_double
        L.fiim_solver_matrix_bytes.restype = C.c_double
        _lib = L
    return _lib


def _check(rc: int):
    if rc != FIIM_OK:
        raise FiimError(rc, lib().fiim_last_error().decode())


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    """ctypes pointer of a numpy array or a torch tensor (host or device), or None."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


# ----------------------------------------------------------------------------- drop-ins
def dropin_cache(enable: bool) -> bool:
    """Device-copy reuse of the drop-ins for this thread (on by default); returns the
    previous setting."""
    return bool(lib().fiim_dropin_cache(C.c_int(1 if enable else 0)))


def EPBiCGSTAB(n, Av, Aj, Ai, b, tol, NMAX, Gv, Gj, Gi, IDv, Hv, Hj, Hi, x, verbose=0):
    """AFIIM EPBiCGSTAB on the GPU. x (float64, C-contiguous) is updated in place."""
    assert x.dtype == np.float64 and x.flags.c_contiguous
    resval, it, info = C.c_double(0), C.c_int(0), C.c_int(-1)
    arrs = [_d(Av), _i(Aj), _i(Ai), _d(b), _d(Gv), _i(Gj), _i(Gi), _d(IDv), _d(Hv), _i(Hj), _i(Hi)]
    _check(lib().fiim_EPBiCGSTAB_afiim(
        C.c_int(n), *[_ptr(a) for a in arrs[:4]], C.c_double(tol), C.c_int(NMAX),
        *[_ptr(a) for a in arrs[4:]], _ptr(x), C.byref(resval), C.byref(it), C.c_int(verbose), C.byref(info)))
    return resval.value, it.value, info.value


def EPBiCGSTAB_pdfiim(A, b, tol, NMAX, G, ID, H, x, issym=False, verbose=0):
    """PDFIIM EPBiCGSTAB. A, G, H are (Ai, Aj, Av) CSR triples; H may be None when issym."""
    assert x.dtype == np.float64 and x.flags.c_contiguous
    Ai, Aj, Av = _i(A[0]), _i(A[1]), _d(A[2])
    Gi, Gj, Gv = _i(G[0]), _i(G[1]), _d(G[2])
    if H is None:
        Hi = Hj = Hv = None
    else:
        Hi, Hj, Hv = _i(H[0]), _i(H[1]), _d(H[2])
    resval, it, info = C.c_double(0), C.c_int(0), C.c_int(-1)
    _check(lib().fiim_EPBiCGSTAB_pdfiim(
        C.c_int(len(Ai) - 1), C.c_int(int(issym)), _ptr(Av), _ptr(Aj), _ptr(Ai), _ptr(_d(b)),
        C.c_double(tol), C.c_int(NMAX), _ptr(Gv), _ptr(Gj), _ptr(Gi), _ptr(_d(ID)), _ptr(Hv), _ptr(Hj),
        _ptr(Hi), _ptr(x), C.byref(resval), C.byref(it), C.c_int(verbose), C.byref(info)))
    return resval.value, it.value, info.value


def PBiCGSTAB(n, Av, Aj, Ai, b, tol, NMAX, Gv, Gj, Gi, IDv, Hv, Hj, Hi, Lv, Lj, Li, Uv, Uj, Ui, nr, mode, x,
              verbose=0):
    """ACIFIM PBiCGSTAB (modes 'E' and 'C')."""
    assert x.dtype == np.float64 and x.flags.c_contiguous
    resval, it, info = C.c_double(0), C.c_int(0), C.c_int(-1)
    lu = [None if a is None else (_i(a) if k % 3 else _d(a)) for k, a in enumerate((Lv, Lj, Li, Uv, Uj, Ui))]
    _check(lib().fiim_PBiCGSTAB_acifim(
        C.c_int(n), _ptr(_d(Av)), _ptr(_i(Aj)), _ptr(_i(Ai)), _ptr(_d(b)), C.c_double(tol), C.c_int(NMAX),
        _ptr(_d(Gv)), _ptr(_i(Gj)), _ptr(_i(Gi)), _ptr(_d(IDv)), _ptr(_d(Hv)), _ptr(_i(Hj)), _ptr(_i(Hi)),
        *[_ptr(a) for a in lu], C.c_int(nr), C.c_char(mode.encode()), _ptr(x), C.byref(resval),
        C.byref(it), C.c_int(verbose), C.byref(info)))
    return resval.value, it.value, info.value


# ----------------------------------------------------------------------------- handle API
class _Handle:
    """A library handle: close() frees it; a with-block closes it on leaving."""

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False


class Solver(_Handle):
    """Set up once (upload, SpMV shape tuning, graph capture); solve many times.

    A: (Ai, Aj, Av); F: dict with Gi, Gj, Gv, IDv, Hi, Hj, Hv (and Li.., Ui.. for mode 'C').
    Arrays are numpy (memory='host') or torch CUDA tensors (memory='device')."""

    def __init__(self, A, F, variant="afiim", issym=False, precision="fp64", mode="E", nr=1,
                 autotune=False, memory="host", verbose=0, inner_tol=1e-5, inner_nmax=1000, max_refine=50,
                 reliable=None):
        self._h = C.c_void_p(0)
        o = Options()
        lib().fiim_options_default(C.byref(o))
        o.variant = _VARIANTS[variant]
        o.issym = int(issym)
        o.precision = _PRECISIONS[precision]
        o.memory = MEM_DEVICE if memory == "device" else MEM_HOST
        o.mode = mode.encode()
        o.nr = nr
        o.autotune = int(autotune)
        o.verbose = verbose
        o.inner_tol = inner_tol
        o.inner_nmax = inner_nmax
        o.max_refine = max_refine
        if reliable is not None:
            o.reliable = reliable
        self.memory = memory
        conv = (lambda a, ints: a) if memory == "device" else (lambda a, ints: None if a is None else (_i(a) if ints else _d(a)))
        self._keep = []

        def P(a, ints):
            a = conv(a, ints)
            self._keep.append(a)
            return _ptr(a)

        g = lambda k: F.get(k)
        n = len(A[0]) - 1
        self.n = n
        _check(lib().fiim_solver_create(
            C.byref(self._h), C.c_int(n), P(A[0], True), P(A[1], True), P(A[2], False),
            P(g("Gi"), True), P(g("Gj"), True), P(g("Gv"), False), P(g("IDv"), False),
            P(g("Hi"), True), P(g("Hj"), True), P(g("Hv"), False),
            P(g("Li"), True), P(g("Lj"), True), P(g("Lv"), False),
            P(g("Ui"), True), P(g("Uj"), True), P(g("Uv"), False), C.byref(o)))
        self._keep = []

    def solve(self, b, x, tol=1e-8, nmax=500) -> dict:
        """x is updated in place; returns the result fields as a dict."""
        r = Result()
        if self.memory != "device":
            b = _d(b)
            assert x.dtype == np.float64 and x.flags.c_contiguous
        _check(lib().fiim_solver_solve(self._h, _ptr(b), _ptr(x), C.c_double(tol), C.c_int(nmax), C.byref(r)))
        return r.as_dict()

    def device_bytes(self) -> int:
        return int(lib().fiim_solver_device_bytes(self._h))

    def spmv_shape(self, which: int):
        """(row-block size, form) of matrix `which` (0 A, 1 G, 2 H): form 0 CSR streams through
        registers, 1 by bulk copies, 2 one warp per row block, 3 the sliced-diagonal copy."""
        t, f = C.c_int(0), C.c_int(0)
        _check(lib().fiim_solver_spmv_shape(self._h, C.c_int(which), C.byref(t), C.byref(f)))
        return t.value, f.value

    def mode(self) -> int:
        """0 device-driven WHILE graph, 1 host-relaunched graph, 2 one cooperative launch, 3 one
        thread-block cluster (the default for systems of at most 32,768 rows)."""
        rc = lib().fiim_solver_mode(self._h)
        if rc < 0:
            _check(rc)
        return rc

    def set_wait_limit(self, polls: int):
        """Bound on each grid-barrier wait of a one-launch solve, in polls (back-to-back acquire
        loads of the barrier word, no sleep between them)."""
        _check(lib().fiim_solver_set_wait_limit(self._h, C.c_int(polls)))

    def test_stall(self):
        """Make the next one-launch solve's first barrier unreachable (it must time out)."""
        _check(lib().fiim_solver_test_stall(self._h))

    def apply(self, x, y, op="A"):
        """y = A x (op 'A') or y = M x (op 'M', the preconditioner) with the solver's kernels."""
        if self.memory != "device":
            x = _d(x)
            assert y.dtype == np.float64 and y.flags.c_contiguous
        _check(lib().fiim_solver_apply(self._h, C.c_int(0 if op == "A" else 1), _ptr(x), _ptr(y)))
        return y

    def kernel_times(self, reps=20, max_kernels=16, in_sequence=False):
        """Mean device ms and algorithmic bytes of each launch of the iteration body, each
        replayed alone; with in_sequence, the body in order with an event between launches,
        returned with the mean ms of the same body without those events."""
        ms, by = np.zeros(max_kernels), np.zeros(max_kernels)
        names = C.create_string_buffer(max_kernels * 32)
        body = C.c_double(0.0)
        if in_sequence:
            k = lib().fiim_solver_kernel_times_seq(self._h, C.c_int(reps), C.c_int(max_kernels), _ptr(ms), _ptr(by),
                                                   names, C.c_int(32), C.byref(body))
        else:
            k = lib().fiim_solver_kernel_times(self._h, C.c_int(reps), C.c_int(max_kernels), _ptr(ms), _ptr(by),
                                               names, C.c_int(32))
        if k < 0:
            _check(k)
        raw = names.raw
        out = [(raw[i * 32:(i + 1) * 32].split(b"\0")[0].decode(), float(ms[i]), float(by[i])) for i in range(k)]
        return (out, body.value) if in_sequence else out

    def iteration_bytes(self) -> float:
        return float(lib().fiim_solver_iteration_bytes(self._h))

    def matrix_bytes(self, which: int) -> float:
        """Bytes one product with matrix `which` reads from it in the form it is served in."""
        return float(lib().fiim_solver_matrix_bytes(self._h, C.c_int(which)))

    def close(self):
        if self._h and self._h.value:
            lib().fiim_solver_destroy(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------------------- row-partitioned solve
def _options(variant="afiim", memory="host", mode="E"):
    o = Options()
    lib().fiim_options_default(C.byref(o))
    o.variant = _VARIANTS[variant]
    o.memory = MEM_DEVICE if memory == "device" else MEM_HOST
    o.mode = mode.encode()
    return o


def dist_partition(A, F, world):
    """Contiguous row blocks balancing the rows' entries of A, G and H (row_starts, int64)."""
    n = len(A[0]) - 1
    rs = np.zeros(world + 1, np.int64)
    Gi = None if F is None else _i(F["Gi"])
    Hi = None if F is None else _i(F["Hi"])
    _check(lib().fiim_dist_partition(C.c_int(n), _ptr(_i(A[0])), _ptr(Gi), _ptr(Hi), C.c_int(world), _ptr(rs)))
    return rs


def dist_rows(M, lo, hi):
    """Rows [lo, hi) of a CSR matrix (rp, ci, v) with global columns, offsets from the block's
    first entry: what rank r is given in a row-partitioned solve."""
    rp, ci, v = M
    e0, e1 = int(rp[lo]), int(rp[hi])
    return _i(np.asarray(rp[lo:hi + 1]) - e0), _i(ci[e0:e1]), _d(v[e0:e1])


def dist_local(A, F, row_starts, rank):
    """Rank `rank`'s rows of A, G, D^{-1} and H."""
    lo, hi = int(row_starts[rank]), int(row_starts[rank + 1])
    Al = dist_rows(A, lo, hi)
    Gl = dist_rows((F["Gi"], F["Gj"], F["Gv"]), lo, hi)
    Hl = dist_rows((F["Hi"], F["Hj"], F["Hv"]), lo, hi)
    Fl = {"Gi": Gl[0], "Gj": Gl[1], "Gv": Gl[2], "IDv": _d(F["IDv"][lo:hi]), "Hi": Hl[0], "Hj": Hl[1], "Hv": Hl[2]}
    return Al, Fl


def dist_plan(rank, world, row_starts, M, fill=0):
    """One matrix's plan on one rank (host only): halo (below, then above), the kept row
    offsets and the renumbered columns. M is the rank's rows (dist_rows)."""
    rs = np.ascontiguousarray(row_starts, dtype=np.int64)
    rp, ci = _i(M[0]), _i(M[1])
    nb, na, nk = C.c_int(0), C.c_int(0), C.c_int(0)
    L = lib()
    _check(L.fiim_dist_plan(C.c_int(rank), C.c_int(world), _ptr(rs), _ptr(rp), _ptr(ci), C.c_int(fill),
                            C.byref(nb), C.byref(na), C.byref(nk), None, None, None))
    halo, krp, cols = np.zeros(nb.value + na.value, np.int32), np.zeros(len(rp), np.int32), np.zeros(nk.value, np.int32)
    _check(L.fiim_dist_plan(C.c_int(rank), C.c_int(world), _ptr(rs), _ptr(rp), _ptr(ci), C.c_int(fill),
                            C.byref(nb), C.byref(na), C.byref(nk), _ptr(halo), _ptr(krp), _ptr(cols)))
    return {"nbelow": nb.value, "nabove": na.value, "halo": halo, "rp": krp, "cols": cols}


def dist_emulate(A, F, b, x, world, tol=1e-8, nmax=1000, variant="afiim", row_starts=None):
    """The row-partitioned solve of `world` row blocks in this process on one GPU (device
    copies in place of NCCL; the same bits as a world-GPU run). x is updated in place."""
    rs = dist_partition(A, F, world) if row_starts is None else np.ascontiguousarray(row_starts, dtype=np.int64)
    n = len(A[0]) - 1
    assert x.dtype == np.float64 and x.flags.c_contiguous
    o = _options(variant)
    r = Result()
    _check(lib().fiim_dist_emulate(
        C.c_int(world), _ptr(rs), C.c_int(n), _ptr(_i(A[0])), _ptr(_i(A[1])), _ptr(_d(A[2])),
        _ptr(_i(F["Gi"])), _ptr(_i(F["Gj"])), _ptr(_d(F["Gv"])), _ptr(_d(F["IDv"])),
        _ptr(_i(F["Hi"])), _ptr(_i(F["Hj"])), _ptr(_d(F["Hv"])), _ptr(_d(b)), _ptr(x),
        C.c_double(tol), C.c_int(nmax), C.byref(o), C.byref(r)))
    return r.as_dict()


def dist_unique_id() -> bytes:
    """NCCL unique id for a DistSolver communicator (make it on one rank, share it)."""
    buf = (C.c_ubyte * 128)()
    _check(lib().fiim_dist_unique_id(buf))
    return bytes(buf)


class DistSolver(_Handle):
    """One rank of a row-partitioned solve (one process per GPU). Collective: every rank
    constructs it with the same uid, world and row_starts, and calls solve together.

    A_local, F_local: this rank's rows (dist_local); b and x of solve: this rank's rows,
    numpy (memory='host') or torch CUDA tensors (memory='device')."""

    def __init__(self, rank, world, uid, row_starts, A_local, F_local, variant="afiim", memory="host", device=-1):
        self._h = C.c_void_p(0)
        self.memory = memory
        o = _options(variant, memory)
        rs = np.ascontiguousarray(row_starts, dtype=np.int64)
        idb = (C.c_ubyte * 128).from_buffer_copy(uid)
        keep = [_i(A_local[0]), _i(A_local[1]), _d(A_local[2]), _i(F_local["Gi"]), _i(F_local["Gj"]),
                _d(F_local["Gv"]), _d(F_local["IDv"]), _i(F_local["Hi"]), _i(F_local["Hj"]), _d(F_local["Hv"])]
        _check(lib().fiim_dist_create(C.byref(self._h), C.c_int(rank), C.c_int(world), idb, C.c_int(device),
                                      _ptr(rs), *[_ptr(a) for a in keep], C.byref(o)))

    def solve(self, b, x, tol=1e-8, nmax=1000) -> dict:
        r = Result()
        if self.memory != "device":
            b = _d(b)
            assert x.dtype == np.float64 and x.flags.c_contiguous
        _check(lib().fiim_dist_solve(self._h, _ptr(b), _ptr(x), C.c_double(tol), C.c_int(nmax), C.byref(r)))
        return r.as_dict()

    def close(self):
        if self._h and self._h.value:
            lib().fiim_dist_destroy(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------------------- sharding
def shard_by_nnz(weights, world, rank):
    """Contiguous shard of independent units (systems, right-hand sides) for `rank` of
    `world`, balanced by weight (e.g. nnz): the cut after unit i lies where the running
    total first reaches (r + 1) / world of the whole. Deterministic, no communication;
    every unit goes to exactly one rank. Returns (first, last) with last exclusive."""
    w = np.asarray(weights, dtype=np.float64)
    if world <= 1 or len(w) == 0:
        return 0, len(w)
    c = np.cumsum(w)
    total = c[-1]
    cuts = [0] + [int(np.searchsorted(c, total * (r + 1) / world, side="left")) + 1 for r in range(world - 1)] + [len(w)]
    cuts = [min(max(x, 0), len(w)) for x in cuts]
    for r in range(1, len(cuts)):
        cuts[r] = max(cuts[r], cuts[r - 1])
    return cuts[rank], cuts[rank + 1]


# ----------------------------------------------------------------------------- batched API
def block_diag(mats):
    """Concatenate CSR triples (Ai, Aj, Av) into one block-diagonal CSR in global numbering.
    Returns ((Ai, Aj, Av), sys_rows)."""
    sizes = [len(m[0]) - 1 for m in mats]
    sys_rows = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    nnz = np.concatenate([[0], np.cumsum([int(m[0][-1]) for m in mats])])
    Ai = np.concatenate([np.asarray(m[0][:-1], np.int64) + nnz[k] for k, m in enumerate(mats)] + [[nnz[-1]]])
    Aj = np.concatenate([np.asarray(m[1], np.int64) + sys_rows[k] for k, m in enumerate(mats)])
    Av = np.concatenate([np.asarray(m[2], np.float64) for m in mats])
    return (Ai.astype(np.int32), Aj.astype(np.int32), Av), sys_rows


class BatchSolver(_Handle):
    """Many independent systems in one device-driven loop (fiim_batch_*).

    systems: list of (A, F) with A = (Ai, Aj, Av) and F = {Gi, Gj, Gv, IDv, Hi, Hj, Hv}.
    precision: 'fp64' | 'fp32' | 'bf16' storage of G and H.
    memory: 'host' (numpy b, x) or 'device' (the concatenated arrays are uploaded here; b, x
    are torch CUDA tensors).
    verified: a system that passes the reference's recurrence test must also have an FP64
    true residual below tol * ||b - A x0||, else it restarts from its current x (at most
    max_restarts rounds); off, the loop stops as the reference's does."""

    def __init__(self, systems, variant="acifim", precision="fp64", memory="host", verified=False,
                 max_restarts=4):
        A, sys_rows = block_diag([s[0] for s in systems])
        G, _ = block_diag([(s[1]["Gi"], s[1]["Gj"], s[1]["Gv"]) for s in systems])
        H, _ = block_diag([(s[1]["Hi"], s[1]["Hj"], s[1]["Hv"]) for s in systems])
        D = np.concatenate([np.asarray(s[1]["IDv"], np.float64) for s in systems])
        self.sys_rows, self.nsys, self.N = sys_rows, len(systems), int(sys_rows[-1])
        self.memory = memory
        o = Options()
        lib().fiim_options_default(C.byref(o))
        o.variant = _VARIANTS[variant]
        o.precision = _PRECISIONS[precision]
        o.memory = MEM_DEVICE if memory == "device" else MEM_HOST
        o.verified = int(verified)
        o.max_restarts = max_restarts
        self._h = C.c_void_p(0)
        arrs = [_i(A[0]), _i(A[1]), _d(A[2]), _i(G[0]), _i(G[1]), _d(G[2]), _d(D), _i(H[0]), _i(H[1]), _d(H[2])]
        if memory == "device":
            import torch
            arrs = [torch.from_numpy(a).cuda() for a in arrs]
        _check(lib().fiim_batch_create(C.byref(self._h), C.c_int(self.nsys), _ptr(_i(sys_rows)),
                                       *[_ptr(a) for a in arrs], C.byref(o)))

    def solve(self, b, x, tol=1e-8, nmax=2000):
        """b, x: concatenated FP64 vectors (x updated in place). Returns per-system arrays."""
        k = self.nsys
        it, info = np.zeros(k, np.int32), np.zeros(k, np.int32)
        rv, tr = np.zeros(k), np.zeros(k)
        r = Result()
        if self.memory != "device":
            b = _d(b)
            assert x.dtype == np.float64 and x.flags.c_contiguous and len(x) == self.N
        _check(lib().fiim_batch_solve(self._h, _ptr(b), _ptr(x), C.c_double(tol), C.c_int(nmax), _ptr(it),
                                      _ptr(info), _ptr(rv), _ptr(tr), C.byref(r)))
        return {"iter": it, "info": info, "resval": rv, "true_relres": tr, "summary": r.as_dict()}

    def close(self):
        if self._h and self._h.value:
            lib().fiim_batch_destroy(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BlockSolver(_Handle):
    """k <= 32 right-hand sides of one system, sharing the sparse products (fiim_block_*).
    B, X: n x k row-major FP64 (numpy, or torch CUDA tensors with memory='device').
    verified: as for BatchSolver, per right-hand side."""

    def __init__(self, A, F, nrhs, variant="afiim", precision="fp64", memory="host", verified=False,
                 max_restarts=4, autotune=False):
        o = Options()
        lib().fiim_options_default(C.byref(o))
        o.autotune = int(autotune)
        o.variant = _VARIANTS[variant]
        o.precision = _PRECISIONS[precision]
        o.memory = MEM_DEVICE if memory == "device" else MEM_HOST
        o.verified = int(verified)
        o.max_restarts = max_restarts
        self.memory, self.k, self.n = memory, nrhs, len(A[0]) - 1
        conv = (lambda a, ints: a) if memory == "device" else (lambda a, ints: _i(a) if ints else _d(a))
        arrs = [conv(A[0], 1), conv(A[1], 1), conv(A[2], 0), conv(F["Gi"], 1), conv(F["Gj"], 1), conv(F["Gv"], 0),
                conv(F["IDv"], 0), conv(F["Hi"], 1), conv(F["Hj"], 1), conv(F["Hv"], 0)]
        self._h = C.c_void_p(0)
        _check(lib().fiim_block_create(C.byref(self._h), C.c_int(self.n), C.c_int(nrhs),
                                       *[_ptr(a) for a in arrs], C.byref(o)))

    def solve(self, B, X, tol=1e-8, nmax=1000):
        k = self.k
        it, info = np.zeros(k, np.int32), np.zeros(k, np.int32)
        rv, tr = np.zeros(k), np.zeros(k)
        r = Result()
        if self.memory != "device":
            B = _d(B)
            assert X.dtype == np.float64 and X.flags.c_contiguous
        _check(lib().fiim_block_solve(self._h, _ptr(B), _ptr(X), C.c_double(tol), C.c_int(nmax), _ptr(it),
                                      _ptr(info), _ptr(rv), _ptr(tr), C.byref(r)))
        return {"iter": it, "info": info, "resval": rv, "true_relres": tr, "summary": r.as_dict()}

    def apply(self, X, Y, op="A"):
        """Y = A X (op 'A') or Y = M X (op 'M') on n x k blocks with the solver's SpMM kernels."""
        if self.memory != "device":
            X = _d(X)
            assert Y.dtype == np.float64 and Y.flags.c_contiguous
        _check(lib().fiim_block_apply(self._h, C.c_int(0 if op == "A" else 1), _ptr(X), _ptr(Y)))
        return Y

    def spmm_shape(self, which):
        """(lanes per row group, right-hand sides per lane) of matrix `which` (0 A, 1 G, 2 H)."""
        lanes, per = C.c_int(0), C.c_int(0)
        _check(lib().fiim_block_spmm_shape(self._h, C.c_int(which), C.byref(lanes), C.byref(per)))
        return lanes.value, per.value

    def close(self):
        if self._h and self._h.value:
            lib().fiim_block_destroy(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------------------- kernel API
def spmv(Ai, Aj, Av, x, y, vec=0, stream=0):
    """y = A x on device tensors (torch CUDA), FP64."""
    _check(lib().fiim_spmv(C.c_int(Ai.numel() - 1), _ptr(Ai), _ptr(Aj), _ptr(Av), _ptr(x), _ptr(y),
                           C.c_int(vec), C.c_void_p(stream)))


def prec_apply(Gi, Gj, Gv, IDv, Hi, Hj, Hv, r, z, tm, stream=0):
    """z = G (IDv o (H r)) on device tensors."""
    _check(lib().fiim_prec_apply(C.c_int(Gi.numel() - 1), _ptr(Gi), _ptr(Gj), _ptr(Gv), _ptr(IDv), _ptr(Hi),
                                 _ptr(Hj), _ptr(Hv), _ptr(r), _ptr(z), _ptr(tm), C.c_void_p(stream)))


def prec_apply_noalloc(Gi, Gj, Gv, IDv, Hi, Hj, Hv, r, z, stream=0):
    """z = G (IDv o (H r)) on device tensors without caller scratch or any allocation
    (the intermediate vector is a fixed array inside the library; n <= 1,048,576)."""
    _check(lib().fiim_prec_apply_noalloc(C.c_int(Gi.numel() - 1), _ptr(Gi), _ptr(Gj), _ptr(Gv), _ptr(IDv),
                                         _ptr(Hi), _ptr(Hj), _ptr(Hv), _ptr(r), _ptr(z), C.c_void_p(stream)))


# ----------------------------------------------------------------------------- generators
def _gen(fn, *args):
    nnz = fn(*args, None, None, None)
    if nnz < 0:
        raise FiimError(FIIM_EARG, "bad generator arguments")
    return nnz


def gen_poisson2d(nx, ny=None):
    ny = nx if ny is None else ny
    L = lib()
    nnz = _gen(L.fiim_gen_poisson2d, C.c_int(nx), C.c_int(ny))
    n = nx * ny
    Ai, Aj, Av = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.fiim_gen_poisson2d(C.c_int(nx), C.c_int(ny), _ptr(Ai), _ptr(Aj), _ptr(Av))
    return Ai, Aj, Av


def gen_convdiff3d(N, peclet=0.5):
    L = lib()
    nnz = _gen(L.fiim_gen_convdiff3d, C.c_int(N), C.c_double(peclet))
    n = N ** 3
    Ai, Aj, Av = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.fiim_gen_convdiff3d(C.c_int(N), C.c_double(peclet), _ptr(Ai), _ptr(Aj), _ptr(Av))
    return Ai, Aj, Av


def gen_convdiff2d(N, diff, theta, peclet):
    L = lib()
    args = (C.c_int(N), C.c_double(diff), C.c_double(theta), C.c_double(peclet))
    nnz = _gen(L.fiim_gen_convdiff2d, *args)
    Ai, Aj, Av = np.zeros(N * N + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.fiim_gen_convdiff2d(*args, _ptr(Ai), _ptr(Aj), _ptr(Av))
    return Ai, Aj, Av


def batch_params(seed, k, side_lo=32, side_hi=256, d_lo=0.1, d_hi=10.0, pe_max=1.0):
    side, diff, theta, pe = C.c_int(0), C.c_double(0), C.c_double(0), C.c_double(0)
    lib().fiim_gen_batch_params(C.c_uint64(seed), C.c_int(k), C.c_int(side_lo), C.c_int(side_hi),
                                C.c_double(d_lo), C.c_double(d_hi), C.c_double(pe_max), C.byref(side),
                                C.byref(diff), C.byref(theta), C.byref(pe))
    return side.value, diff.value, theta.value, pe.value


def zipf_scale(n, alpha=2.0, cap=512, mean=16.0, seed=20261203, sample=200000):
    """Scale of the Zipf draws that gives the target mean row length (bisection)."""
    L = lib()
    lo, hi = 0.5, 64.0
    for _ in range(40):
        mid = 0.5 * (lo + hi)
        m = L.fiim_gen_zipf_mean(C.c_int(n), C.c_double(alpha), C.c_int(cap), C.c_double(mid),
                                 C.c_uint64(seed), C.c_int(sample))
        if m < mean:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def gen_zipf(n, scale, alpha=2.0, cap=512, seed=20261203):
    L = lib()
    args = (C.c_int(n), C.c_double(alpha), C.c_int(cap), C.c_double(scale), C.c_uint64(seed))
    nnz = _gen(L.fiim_gen_zipf, *args)
    Ai, Aj, Av = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.fiim_gen_zipf(*args, _ptr(Ai), _ptr(Aj), _ptr(Av))
    return Ai, Aj, Av


def rand_normal(n, seed):
    out = np.zeros(n)
    lib().fiim_rand_normal(C.c_long(n), C.c_uint64(seed), _ptr(out))
    return out


def model_rhs(A):
    Ai, Aj, Av = _i(A[0]), _i(A[1]), _d(A[2])
    b = np.zeros(len(Ai) - 1)
    lib().fiim_model_rhs(C.c_int(len(Ai) - 1), _ptr(Ai), _ptr(Aj), _ptr(Av), _ptr(b))
    return b


def pdfiim_build(A, ftol, prefill=1, lfill=1, postfill=1, warpsize=-1, filttype="I", patt="B", gpu=False):
    """PDFIIM construction (same factors as PDFIIM/src/parPrec.cpp:95-588), on the host or,
    with gpu=True, on the GPU (the same factors bit for bit). Returns a factor dict."""
    Ai, Aj, Av = _i(A[0]), _i(A[1]), _d(A[2])
    n = len(Ai) - 1
    ng, nh = C.c_int(0), C.c_int(0)
    L = lib()
    fn = L.fiim_pdfiim_build_gpu if gpu else L.fiim_pdfiim_build
    args = (C.c_int(n), _ptr(Ai), _ptr(Aj), _ptr(Av), C.c_int(prefill), C.c_int(lfill), C.c_int(postfill),
            C.c_double(ftol), C.c_int(warpsize), C.c_char(filttype.encode()), C.c_char(patt.encode()))
    rc = fn(*args, C.byref(ng), C.byref(nh), None, None, None, None, None, None, None)
    if rc != FIIM_OK:
        if gpu:
            _check(rc)
        raise FiimError(rc, "pdfiim_build rejected its arguments")
    F = {"Gv": np.zeros(ng.value), "Gj": np.zeros(ng.value, np.int32), "Gi": np.zeros(n + 1, np.int32),
         "IDv": np.zeros(n), "Hv": np.zeros(nh.value), "Hj": np.zeros(nh.value, np.int32),
         "Hi": np.zeros(n + 1, np.int32)}
    _check(fn(*args, C.byref(ng), C.byref(nh), _ptr(F["Gv"]), _ptr(F["Gj"]), _ptr(F["Gi"]),
                               _ptr(F["IDv"]), _ptr(F["Hv"]), _ptr(F["Hj"]), _ptr(F["Hi"])))
    return F


def afiim_build(A, dtol, elem_per_rowcol=10, growth=5, eta=0.0, shift=0.0):
    """AFIIM construction on the host (the same factors as AFIIM/src/prec.cpp:101-767; the
    defaults are the example driver's, AFIIM/example/example.cpp:37-39). Returns a factor
    dict. Sequential in the rows; safe to call from several threads."""
    Ai, Aj, Av = _i(A[0]), _i(A[1]), _d(A[2])
    n = len(Ai) - 1
    ng, nh = C.c_int(0), C.c_int(0)
    L = lib()
    args = (C.c_int(n), _ptr(Ai), _ptr(Aj), _ptr(Av), C.c_double(dtol), C.c_int(elem_per_rowcol), C.c_int(growth),
            C.c_double(eta), C.c_double(shift), C.byref(ng), C.byref(nh))
    _check(L.fiim_afiim_build(*args, *([None] * 7)))
    F = {"Gv": np.zeros(ng.value), "Gj": np.zeros(ng.value, np.int32), "Gi": np.zeros(n + 1, np.int32),
         "IDv": np.zeros(n), "Hv": np.zeros(nh.value), "Hj": np.zeros(nh.value, np.int32),
         "Hi": np.zeros(n + 1, np.int32)}
    _check(L.fiim_afiim_build(*args, *[_ptr(F[k]) for k in ("Gv", "Gj", "Gi", "IDv", "Hv", "Hj", "Hi")]))
    return F


def acifim_build(A, dtol1, dtol2, elem_per_rowcol=30, growth=5, eta=0.0, shift=0.0, coeff=2.0,
                 element_limit=200, filtit=30, with_lu=False):
    """ACIFIM construction on the host (the same factors as ACIFIM/src/prec.cpp:127-1052; the
    defaults are the example driver's, ACIFIM/example/example.cpp:42-47). Returns a factor
    dict (with Li.., Ui.. when with_lu). Raises FiimError when the construction fails (a NaN
    Schur complement, where the reference returns 1). Safe to call from several threads."""
    Ai, Aj, Av = _i(A[0]), _i(A[1]), _d(A[2])
    n = len(Ai) - 1
    nnz = np.zeros(4, np.int32)
    L = lib()
    args = (C.c_int(n), _ptr(Ai), _ptr(Aj), _ptr(Av), C.c_double(dtol1), C.c_double(dtol2), C.c_int(elem_per_rowcol),
            C.c_int(growth), C.c_double(eta), C.c_double(shift), C.c_double(coeff), C.c_int(element_limit),
            C.c_int(filtit), _ptr(nnz))
    _check(L.fiim_acifim_build(*args, *([None] * 13)))
    ng, nh, nl, nu = (int(v) for v in nnz)
    F = {"Gv": np.zeros(ng), "Gj": np.zeros(ng, np.int32), "Gi": np.zeros(n + 1, np.int32), "IDv": np.zeros(n),
         "Hv": np.zeros(nh), "Hj": np.zeros(nh, np.int32), "Hi": np.zeros(n + 1, np.int32)}
    if with_lu:
        F.update({"Lv": np.zeros(nl), "Lj": np.zeros(nl, np.int32), "Li": np.zeros(n + 1, np.int32),
                  "Uv": np.zeros(nu), "Uj": np.zeros(nu, np.int32), "Ui": np.zeros(n + 1, np.int32)})
    keys = ("Gv", "Gj", "Gi", "IDv", "Hv", "Hj", "Hi", "Lv", "Lj", "Li", "Uv", "Uj", "Ui")
    _check(L.fiim_acifim_build(*args, *[_ptr(F.get(k)) for k in keys]))
    return F


def read_mtx(path, form="afiim"):
    """Matrix Market matrix -> ((Ai, Aj, Av), issym), the same arrays as the reference's
    reader: form 'afiim' (also ACIFIM) expands a symmetric file, 'pdfiim' keeps its upper
    triangle and returns issym = True."""
    n, z, sym = C.c_int(0), C.c_int(0), C.c_int(0)
    f = 1 if form == "pdfiim" else 0
    _check(lib().fiim_read_mtx(os.fsencode(path), C.c_int(f), C.byref(n), C.byref(z), C.byref(sym),
                               None, None, None))
    Ai, Aj, Av = np.zeros(n.value + 1, np.int32), np.zeros(z.value, np.int32), np.zeros(z.value)
    _check(lib().fiim_read_mtx(None, C.c_int(f), C.byref(n), C.byref(z), C.byref(sym), _ptr(Ai), _ptr(Aj),
                               _ptr(Av)))
    return (Ai, Aj, Av), bool(sym.value)


def read_rhs(path):
    n = C.c_int(0)
    _check(lib().fiim_read_rhs(os.fsencode(path), C.c_int(0), None, C.byref(n)))
    b = np.zeros(n.value)
    _check(lib().fiim_read_rhs(os.fsencode(path), C.c_int(n.value), _ptr(b), C.byref(n)))
    return b


def factors_save(path, F):
    """Writes G, D^{-1}, H of a factor dict (Gi, Gj, Gv, IDv, Hi, Hj, Hv) to a binary file."""
    Gi, Gj, Gv = _i(F["Gi"]), _i(F["Gj"]), _d(F["Gv"])
    Hi, Hj, Hv = _i(F["Hi"]), _i(F["Hj"]), _d(F["Hv"])
    _check(lib().fiim_factors_save(os.fsencode(path), C.c_int(len(Gi) - 1), _ptr(Gi), _ptr(Gj), _ptr(Gv),
                                   _ptr(_d(F["IDv"])), _ptr(Hi), _ptr(Hj), _ptr(Hv)))


def factors_load(path):
    n, ng, nh = C.c_int(0), C.c_int(0), C.c_int(0)
    L = lib()
    _check(L.fiim_factors_load(os.fsencode(path), C.byref(n), C.byref(ng), C.byref(nh), None, None, None, None,
                               None, None, None))
    F = {"Gi": np.zeros(n.value + 1, np.int32), "Gj": np.zeros(ng.value, np.int32), "Gv": np.zeros(ng.value),
         "IDv": np.zeros(n.value), "Hi": np.zeros(n.value + 1, np.int32), "Hj": np.zeros(nh.value, np.int32),
         "Hv": np.zeros(nh.value)}
    _check(L.fiim_factors_load(None, C.byref(n), C.byref(ng), C.byref(nh), *[_ptr(F[k]) for k in
                               ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")]))
    return F


@dataclass
class Problem:
    """A generated system with its factors, as the benches and tests use it."""
    A: tuple
    b: np.ndarray
    F: dict
    name: str
