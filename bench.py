"""Benchmark of the preconditioned BiCGSTAB solve phase on B200.

Workload (one GPU): 3D 7-point upwind convection-diffusion on a 128^3 grid (n = 2,097,152,
nnz = 14,581,760), unit diffusion, cell Peclet 0.5, b ~ N(0,1) (seed 20261203), x0 = 0,
PDFIIM factors eps 0.05 (prefill 2, lfill 2, postfill 1, no warpsize limit, inf-norm filter,
both-triangle pattern) built by the library's host construction, FP64 BiCGSTAB to 1e-8,
NMAX 1200. A step is one full solve. Synthetic data (the reference names no dataset).

  value  solves/s with A, G, D^-1, H, b resident in HBM (handle API, device arrays),
         device time of each solve call (CUDA events on the solver's stream)
  e2e    solves/s through the reference-facing C-ABI call fiim_EPBiCGSTAB_pdfiim with
         pinned host arrays: every step uploads A, G, D^-1, H, b, x0 and downloads x
         (host wall clock around the blocking call). e2e.same_system_new_rhs: the same
         call with a new b each step and the call's device-copy reuse on (content hash of
         every matrix array each call; only b and x0 uploaded)

--impl reference times the reference's own EPBiCGSTAB (oracle/_ref: the reference's
sources compiled against the project's MKL shim, OpenMP on all host cores) on the same
system, built with numpy (no library of this project is loaded), with the reference's own
pdfiim factors; each step is one full solve, the EPBiCGSTAB call alone timed.

Multi-GPU (torchrun): by default one full replica per rank (nothing is exchanged during a
solve), value = total solves / max-over-ranks time, weak scaling. --partition rows splits the
one system into row blocks over the ranks instead (NCCL halo exchange and gathered partial
sums each iteration), value = solves of the whole system / max-over-ranks time, strong
scaling. At N = 1 the "partitioned" leg runs that path on one rank.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "computational-mathematics_b200")
ORACLE = os.path.join(ROOT, "oracle")
sys.path.insert(0, PKG)

METRIC = "BiCGSTAB solves/sec to 1e-8 rel. residual + HBM GB/s; mixed/batched vs FP64"
SEED = 20261203
PDFIIM_PARAMS = dict(ftol=0.05, prefill=2, lfill=2, postfill=1, warpsize=-1, filttype="I", patt="B")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload(N):
    import fiim_b200 as FB
    A = FB.gen_convdiff3d(N, 0.5)
    b = FB.rand_normal(N ** 3, SEED)
    return A, b


# The same system built without the library, for the reference arm: a process that times the
# reference maps none of this project's code. Both restate fiim_gen.cpp (fiim_gen_convdiff3d,
# fiim_rand_normal) operation for operation, so the arrays are the library's bit for bit
# (tests/test_bench_contract.py compares them).
_U64 = np.uint64


def _splitmix64(s):
    """Returns (advanced state, output) of splitmix64 on a uint64 array (wrapping arithmetic)."""
    s = s + _U64(0x9E3779B97F4A7C15)
    z = s
    z = (z ^ (z >> _U64(30))) * _U64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> _U64(27))) * _U64(0x94D049BB133111EB)
    return s, z ^ (z >> _U64(31))


def rand_normal_host(n, seed):
    """fiim_rand_normal: stream i is seeded from (seed, i); Box-Muller of its next two draws.
    log and cos are libm's, through the math module, as the library calls them."""
    import math
    idx = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        s = _U64(seed) ^ (_U64(0xD1B54A32D192ED03) * (idx + _U64(1)))
        s, _ = _splitmix64(s)
        s, z1 = _splitmix64(s)
        s, z2 = _splitmix64(s)
    u1 = (z1 >> _U64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    u2 = (z2 >> _U64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    u1 = np.where(u1 < 1e-300, 1e-300, u1)
    log, cos, sqrt = math.log, math.cos, math.sqrt
    return np.array([sqrt(-2.0 * log(a)) * cos(6.283185307179586 * c) for a, c in zip(u1.tolist(), u2.tolist())])


def convdiff3d_host(N, peclet=0.5):
    """fiim_gen_convdiff3d: 7-point upwind convection-diffusion, entries of a row in the
    order z-1, y-1, x-1, diagonal, x+1, y+1, z+1."""
    n, NN = N ** 3, N * N
    i = np.arange(n, dtype=np.int64)
    x, y, z = i % N, (i // N) % N, i // NN
    keep = np.stack([z > 0, y > 0, x > 0, np.ones(n, bool), x < N - 1, y < N - 1, z < N - 1], axis=1)
    cols = i[:, None] + np.array([-NN, -N, -1, 0, 1, N, NN], np.int64)[None, :]
    lo, hi = -1.0 - peclet, -1.0
    vals = np.broadcast_to(np.array([lo, lo, lo, 6.0 + 3.0 * peclet, hi, hi, hi]), (n, 7))
    Ai = np.zeros(n + 1, np.int32)
    Ai[1:] = np.cumsum(keep.sum(axis=1))
    return Ai, cols[keep].astype(np.int32), vals[keep].copy()


def workload_host(N):
    return convdiff3d_host(N, 0.5), rand_normal_host(N ** 3, SEED)


def repo_libraries():
    """Shared objects of this repository mapped into this process (from /proc/self/maps)."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") and path.startswith(ROOT + os.sep):
                    out.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(out)


def config(N, nnz):
    """The workload, identical in both arms' lines."""
    return {"workload": f"convdiff3d_{N} (n={N ** 3:,}, nnz={nnz:,}) PDFIIM eps 0.05 (2,2,1) FP64 BiCGSTAB",
            "n": N ** 3, "nnz": int(nnz), "tol": 1e-8, "nmax": 1200,
            "l2": "inputs larger than L2 (A+G+H+vectors >> 126 MB), no flush"}


class Clocks:
    """nvidia-smi samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def __enter__(self):
        # The sampler is started, and its first sample awaited, before the timed region: the
        # start-up of nvidia-smi slows kernel launches for a moment.
        self.lines = []
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
            return self
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()
        t0 = time.time()
        while not self.lines and time.time() - t0 < 5.0 and self.p.poll() is None:
            time.sleep(0.02)
        time.sleep(0.3)
        self.skip = len(self.lines)
        return self

    def _read(self):
        for line in self.p.stdout:
            if line.strip():
                self.lines.append(line)

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.reader.join(timeout=5)
            # keep the samples taken during the timed region (the warm-up ones, too, if
            # the region was shorter than one sampling period)
            self.lines = self.lines[self.skip:] or self.lines

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(backend="nccl"):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE); NCCL for the barrier
    and the max over ranks. backend 'gloo' is the CPU dry run of the launcher."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws == 1:
        return 0, 1, None
    import datetime
    import torch
    import torch.distributed as dist
    rank, local = int(os.environ["RANK"]), int(os.environ.get("LOCAL_RANK", "0"))
    if backend == "gloo":
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    else:
        if local >= torch.cuda.device_count():
            raise SystemExit(f"rank {rank}: local rank {local} but only {torch.cuda.device_count()} GPUs visible")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    print(f"bench: rank {rank} of {ws} ({backend}, local rank {local})", file=sys.stderr, flush=True)
    return rank, ws, dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cpu" if dist.get_backend() == "gloo" else "cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def launch_ranks(args):
    """`bench.py --gpus N` started without torchrun: start the N ranks on this node (one process
    per GPU, rendezvous on 127.0.0.1) with the same arguments, and return their status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    print("bench: starting " + " ".join(cmd), file=sys.stderr, flush=True)
    return subprocess.call(cmd)


def run_dry(args):
    """The launcher and timing protocol without a GPU (gloo): every rank runs W untimed and K
    timed steps between barriers, rank r's step lasting (r + 1) x 10 ms, and rank 0 prints the
    max over ranks. Nothing is solved: the line says dry_run and carries no metric."""
    rank, ws, dist = dist_init("gloo")
    step = lambda: time.sleep(0.01 * (rank + 1))
    for _ in range(args.warmup):
        step()
    barrier(dist)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    mine = time.perf_counter() - t0
    barrier(dist)
    worst = max_over_ranks(dist, mine)
    if rank == 0:
        print(json.dumps({"dry_run": True, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1000 * worst / args.steps, "rank0_ms_per_step": 1000 * mine / args.steps}),
              flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------- CPU reference
def cpu_kind():
    """'reference' when the reference compiled against the MKL shim is present (oracle/_ref),
    else 'port' (the plain-C restatement, one thread)."""
    sys.path.insert(0, ORACLE)
    import pyoracle as O
    if O.have_ref("pdfiim"):
        return "reference"
    subprocess.run(["make", "-s", "-C", ORACLE, "restatement"], check=True)
    return "port"


class CpuSolves:
    """Full solves of the benchmark system by the reference's own EPBiCGSTAB
    (PDFIIM/src/bicgstab.cpp:80-310, OpenMP on every host core through the MKL shim), with the
    reference's own pdfiim factors (PDFIIM/src/parPrec.cpp:95-588). The system is held as the
    reference's sparseMatrix objects, built once: each step times the EPBiCGSTAB call alone.
    Without oracle/_ref, the restatement (one thread) stands in, on a bounded sample of
    `port_its` iterations scaled to a full solve's count (a full 1-thread solve takes minutes)."""

    def __init__(self, A, b, port_its=12):
        sys.path.insert(0, ORACLE)
        import pyoracle as O
        self.O, self.A, self.b, self.port_its = O, A, b, port_its
        self.kind = cpu_kind()
        t0 = time.perf_counter()
        if self.kind == "reference":
            self.threads = os.cpu_count() or 1
            O.set_threads(self.threads, "pdfiim")
            self.F = O.pdfiim_build(A, **PDFIIM_PARAMS)
            self.sys = O.RefPdfiimSystem(A, self.F)
        else:
            self.threads = 1
            self.F = None
        self.setup_s = time.perf_counter() - t0
        self.its_full = None

    def factors(self):
        return self.F

    def step(self):
        """One step: (seconds, iterations, info, x); a full solve (reference) or the sample."""
        if self.kind == "reference":
            x, res, it, info, secs = self.sys.run(self.b, tol=1e-8, nmax=1200)
            self.its_full = it
            return secs, it, info, x
        if self.F is None:
            # the port has no construction of its own: the reference's factors equal the
            # library's bit for bit (tests/test_host.py), so the port uses those
            import fiim_b200 as FB
            self.F = FB.pdfiim_build(self.A, **PDFIIM_PARAMS)
        t0 = time.perf_counter()
        x, res, it, info = self.O.bicgstab("pdfiim", self.A, self.b, self.F, tol=1e-8, nmax=self.port_its)
        dt = time.perf_counter() - t0
        return dt, it, info, x

    def describe(self, steps, its_full, dt_total):
        if self.kind == "reference":
            return (f"{steps} full solves of the {len(self.b):,}-row system ({its_full} iterations each, "
                    f"{dt_total:.1f} s), the EPBiCGSTAB call alone timed; sparseMatrix objects built once")
        return (f"{steps} x {self.port_its} iterations of the restatement (one thread, {dt_total:.1f} s), "
                f"scaled by a full solve's {its_full} iterations")

    def close(self):
        if self.kind == "reference":
            self.sys.close()


def run_reference(args):
    """The reference arm: the reference's own CPU solve on this box's host cores. It builds the
    system with numpy (workload_host), so this process maps no library of this project."""
    rank = int(os.environ.get("RANK", "0"))
    ws = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    if rank != 0:
        return 0
    A, b = workload_host(args.size)
    nnz = int(A[0][-1])
    cs = CpuSolves(A, b)
    for _ in range(args.warmup):
        cs.step()
    secs, its, infos = [], [], []
    for _ in range(args.steps):
        s, it, info, _ = cs.step()
        secs.append(s)
        its.append(it)
        infos.append(info)
    if cs.kind == "reference":
        its_full, tot = int(np.median(its)), sum(secs)
    else:
        # the port's samples stop at port_its; a full solve takes the reference's 99 on this system
        its_full, tot = 99, sum(s * 99 / max(it, 1) for s, it in zip(secs, its))
    v = args.steps / tot
    cs.close()
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config(args.size, nnz),
            "iterations": its_full, "info": infos[-1], "setup_s": round(cs.setup_s, 2),
            "parallelism": f"host, {cs.threads} OpenMP threads",
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cs.threads, "kind": cs.kind,
                             "sample": cs.describe(args.steps, its_full, sum(secs))},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "libraries_loaded": repo_libraries()}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------- GPU arm
def run_e2e(args, A, F, b, n, ws, dist):
    """Steps through fiim_EPBiCGSTAB_pdfiim with pinned host arrays (uploads and download inside)."""
    import torch
    import fiim_b200 as FB
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hA = [pin(a) for a in A]
    hG = [pin(F[k]) for k in ("Gi", "Gj", "Gv")]
    hH = [pin(F[k]) for k in ("Hi", "Hj", "Hv")]
    hD, hb = pin(F["IDv"]), pin(b)
    hx = torch.zeros(n, dtype=torch.float64).pin_memory()
    L = FB.lib()
    resval, it, info = C.c_double(0), C.c_int(0), C.c_int(0)
    P = lambda t: C.c_void_p(t.data_ptr())

    def e2e_call(rhs):
        rc = L.fiim_EPBiCGSTAB_pdfiim(C.c_int(n), 0, P(hA[2]), P(hA[1]), P(hA[0]), P(rhs), C.c_double(1e-8), 1200,
                                      P(hG[2]), P(hG[1]), P(hG[0]), P(hD), P(hH[2]), P(hH[1]), P(hH[0]), P(hx),
                                      C.byref(resval), C.byref(it), 0, C.byref(info))
        FB._check(rc)

    def timed(rhs_list):
        for k in range(args.warmup):
            hx.zero_()
            e2e_call(rhs_list[k % len(rhs_list)])
        barrier(dist)
        e_times = []
        for k in range(args.steps):
            hx.zero_()                      # the caller's initial guess, x0 = 0
            t1 = time.perf_counter()        # timed: the C-ABI call alone
            e2e_call(rhs_list[k % len(rhs_list)])
            e_times.append(time.perf_counter() - t1)
        return max_over_ranks(dist, sum(e_times))

    # Headline: every step uploads the whole system (the drop-in's device-copy reuse is off).
    prev = FB.dropin_cache(False)
    e_tot = timed([hb])
    h2d = sum(int(t.numel() * t.element_size()) for t in hA + hG + hH + [hD, hb, hx])
    out = {"value": args.steps * ws / e_tot, "unit": "solves/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": 8 * n, "timing": "host wall clock around the blocking call",
           "device_copies": "all inputs uploaded every step", "iter": it.value, "info": info.value}
    # The same call with pageable host arrays (plain numpy memory, as the reference's drivers
    # pass std::vector data), everything uploaded every step.
    pg = {"A": [np.ascontiguousarray(a) for a in A], "G": [np.ascontiguousarray(F[k]) for k in ("Gi", "Gj", "Gv")],
          "H": [np.ascontiguousarray(F[k]) for k in ("Hi", "Hj", "Hv")], "D": np.ascontiguousarray(F["IDv"]),
          "b": np.ascontiguousarray(b), "x": np.zeros(n)}
    Pn = lambda a: a.ctypes.data_as(C.c_void_p)

    def pageable_call():
        rc = L.fiim_EPBiCGSTAB_pdfiim(C.c_int(n), 0, Pn(pg["A"][2]), Pn(pg["A"][1]), Pn(pg["A"][0]), Pn(pg["b"]),
                                      C.c_double(1e-8), 1200, Pn(pg["G"][2]), Pn(pg["G"][1]), Pn(pg["G"][0]),
                                      Pn(pg["D"]), Pn(pg["H"][2]), Pn(pg["H"][1]), Pn(pg["H"][0]), Pn(pg["x"]),
                                      C.byref(resval), C.byref(it), 0, C.byref(info))
        FB._check(rc)

    for _ in range(args.warmup):
        pg["x"][:] = 0.0
        pageable_call()
    barrier(dist)
    p_times = []
    for _ in range(args.steps):
        pg["x"][:] = 0.0
        t1 = time.perf_counter()
        pageable_call()
        p_times.append(time.perf_counter() - t1)
    p_tot = max_over_ranks(dist, sum(p_times))
    out["pageable_host_arrays"] = {"value": args.steps * ws / p_tot, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                                   "d2h_bytes_per_step": 8 * n,
                                   "device_copies": "all inputs uploaded every step from pageable memory"}
    # The same system with a new right-hand side each step and the reuse on (the default):
    # each call hashes A, G, D^-1, H (content stamps) and uploads only b and x0.
    FB.dropin_cache(True)
    rhs = [pin(FB.rand_normal(n, 20261203 + 1 + k)) for k in range(4)]
    e_tot2 = timed(rhs)
    FB.dropin_cache(prev)
    out["same_system_new_rhs"] = {
        "value": args.steps * ws / e_tot2, "unit": "solves/s", "h2d_bytes_per_step": 16 * n,
        "d2h_bytes_per_step": 8 * n, "device_copies": "matrices reused after a content-hash check of every array",
        "iter_last": it.value, "info_last": info.value}
    return out



def run_small(args, dev):
    """The small plain case (2D 5-point Poisson on a 128 x 128 grid, n = 16,384, b = A 1,
    x0 = 0, AFIIM factors with drop tolerance 0.1, FP64, rtol 1e-8, NMAX 1000). The factors
    are the ones the reference built for the committed fixture tests/golden/poisson128_afiim.npz
    (data only). The working set fits in L2: the solve is bound by launch and reduction latency,
    not HBM bandwidth. The default path at this size is one thread-block cluster (the solve
    vectors in the CTAs' shared memory); the WHILE graph and the cooperative launch are timed
    beside it."""
    import torch
    import fiim_b200 as FB
    z = np.load(os.path.join(ROOT, "tests", "golden", "poisson128_afiim.npz"))
    A = tuple(torch.from_numpy(z[k]).to(dev) for k in ("Ai", "Aj", "Av"))
    F = {k: torch.from_numpy(z[k]).to(dev) for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}
    b = torch.from_numpy(z["b"]).to(dev)
    x = torch.zeros_like(b)
    def timed(persist):
        prev = os.environ.get("FIIM_PERSIST")
        if persist is None:
            os.environ.pop("FIIM_PERSIST", None)
        else:
            os.environ["FIIM_PERSIST"] = persist
        try:
            S = FB.Solver(A, F, variant="afiim", memory="device")
        finally:
            if prev is None:
                os.environ.pop("FIIM_PERSIST", None)
            else:
                os.environ["FIIM_PERSIST"] = prev
        mode = S.mode()
        for _ in range(max(args.warmup, 3)):
            x.zero_()
            S.solve(b, x, tol=1e-8, nmax=1000)
        rr = []
        for _ in range(max(args.steps, 20)):
            x.zero_()
            rr.append(S.solve(b, x, tol=1e-8, nmax=1000))
        S.close()
        ms = sum(q["device_ms"] for q in rr) / len(rr)
        return {"solves_per_s": round(1000.0 / ms, 2), "ms_per_solve": round(ms, 4), "iterations": rr[-1]["iter"],
                "us_per_iteration": round(1000.0 * ms / max(rr[-1]["iter"], 1), 2), "info": rr[-1]["info"],
                "mode": {0: "WHILE graph", 1: "host-relaunched graph", 2: "one cooperative launch",
                         3: "one thread-block cluster"}[mode]}
    out = {"workload": "poisson2d_128 (n=16,384) AFIIM eps 0.1 (reference-built factors) FP64 BiCGSTAB",
           "reference_iterations": int(z["iter"]), "reference_iteration_envelope": [int(v) for v in z["iter_env"]],
           "bound": "latency (working set in L2)"}
    out.update(timed(None))                  # the default: one thread-block cluster at this size
    out["while_graph"] = timed("0")
    out["one_cooperative_launch"] = timed("1")
    return out


def run_partitioned(args, A, F, b, rank, ws, dist, dev):
    """The system split into ws contiguous row blocks, one per rank (fiim_dist_*: NCCL halo
    exchange before each product, gathered partial sums for the scalars). Strong scaling:
    one solve of the whole system per step, value = steps / max-over-ranks device time.
    At ws = 1 it measures the partition machinery's own cost (NCCL at one rank, one-thread
    scalar kernels, host-relaunched graph) against the single-GPU solve."""
    import torch
    import fiim_b200 as FB
    rs = FB.dist_partition(A, F, ws)
    uid = [FB.dist_unique_id() if rank == 0 else None]
    if dist is not None:
        dist.broadcast_object_list(uid, src=0)
    lo, hi = int(rs[rank]), int(rs[rank + 1])
    Al, Fl = FB.dist_local(A, F, rs, rank)
    D = FB.DistSolver(rank, ws, uid[0], rs, Al, Fl, variant="pdfiim", memory="device", device=dev.index)
    bl = torch.from_numpy(np.ascontiguousarray(b[lo:hi])).to(dev)
    xl = torch.zeros(hi - lo, dtype=torch.float64, device=dev)
    for _ in range(args.warmup):
        xl.zero_()
        D.solve(bl, xl, tol=1e-8, nmax=1200)
    torch.cuda.synchronize()
    barrier(dist)
    rr = []
    for _ in range(args.steps):
        xl.zero_()
        rr.append(D.solve(bl, xl, tol=1e-8, nmax=1200))
    torch.cuda.synchronize()
    dev_ms = max_over_ranks(dist, sum(q["device_ms"] for q in rr))
    assert all(q["info"] == 0 for q in rr), rr[0]
    # e2e: the same call with this rank's b and x in pinned host memory (copies inside).
    hb = torch.from_numpy(np.ascontiguousarray(b[lo:hi])).pin_memory()
    hx = torch.zeros(hi - lo, dtype=torch.float64).pin_memory()
    D.close()
    uid2 = [FB.dist_unique_id() if rank == 0 else None]
    if dist is not None:
        dist.broadcast_object_list(uid2, src=0)
    Dh = FB.DistSolver(rank, ws, uid2[0], rs, Al, Fl, variant="pdfiim", memory="host", device=dev.index)
    for _ in range(args.warmup):
        hx.zero_()
        Dh.solve(hb.numpy(), hx.numpy(), tol=1e-8, nmax=1200)
    barrier(dist)
    e_times = []
    for _ in range(args.steps):
        hx.zero_()
        t1 = time.perf_counter()
        Dh.solve(hb.numpy(), hx.numpy(), tol=1e-8, nmax=1200)
        e_times.append(time.perf_counter() - t1)
    e_tot = max_over_ranks(dist, sum(e_times))
    Dh.close()
    return {"value": args.steps / (dev_ms / 1000.0), "unit": "solves/s", "ms_per_solve": dev_ms / args.steps,
            "ranks": ws, "row_starts": [int(v) for v in rs], "iterations": rr[-1]["iter"],
            "true_relres": rr[-1]["true_relres"], "launches_per_solve_per_rank": rr[-1]["launches"],
            "e2e": {"value": args.steps / e_tot, "unit": "solves/s", "h2d_bytes_per_step": 16 * (hi - lo),
                    "d2h_bytes_per_step": 8 * (hi - lo), "bytes": "of rank 0's rows",
                    "timing": "host wall clock around the blocking call, max over ranks"}}


def run_batched(args, rank=0, world=1, dist=None):
    """256 independent 2D convection-diffusion systems (side U{32..256}, diffusion log-U[0.1,10],
    random direction, cell Peclet <= 1), each with ACIFIM factors (eps1 0.1, eps2 0.05, the
    example driver's other parameters) from the library's construction (the reference's
    acifim, bit for bit; one system per host thread), solved (a) in one batched launch with
    FP32 factor storage, (b) the same with FP64 factors, both FP64-verified, (c) FP32 factors
    stopped on the reference's recurrence test alone, and (d) one after another with the FP64
    single-system solver. Loop control: ACIFIM's (divergence window 40, non-finite-alpha
    guard), mode 'E'."""
    from concurrent.futures import ThreadPoolExecutor
    import torch
    import fiim_b200 as FB
    # Systems are independent: with N ranks each solves a contiguous, nnz-balanced shard
    # (no exchange on the data path); the whole-job rate divides all systems by the
    # max-over-ranks time.
    sides = [FB.batch_params(SEED, k)[0] for k in range(args.batch)]
    lo, hi = FB.shard_by_nnz([5 * s * s for s in sides], world, rank)

    def one(k):
        side, diff, theta, pe = FB.batch_params(SEED, k)
        A = FB.gen_convdiff2d(side, diff, theta, pe)
        return A, FB.acifim_build(A, 0.1, 0.05), FB.rand_normal(side * side, SEED + 10 + k)

    t0 = time.perf_counter()
    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        systems = list(ex.map(one, range(lo, hi)))
    setup = time.perf_counter() - t0
    b = np.concatenate([s[2] for s in systems])
    N = len(b)
    out = {"systems": len(systems), "rows": N, "nnz": int(sum(int(s[0][0][-1]) for s in systems)),
           "factor_nnz": int(sum(len(s[1]["Gv"]) + len(s[1]["Hv"]) for s in systems)),
           "tol": 1e-8, "loop": "ACIFIM", "factors": "ACIFIM eps1 0.1 eps2 0.05, library construction "
                                                     "(the reference's acifim bit for bit)",
           "setup_s": round(setup, 2),
           "verified": "FP64 true residual of every system below tol (masked restarts from x)"}
    # Inputs resident in HBM, as for the headline value: b and x are device arrays.
    tb = torch.from_numpy(b).cuda()
    tx = torch.zeros(N, dtype=torch.float64, device="cuda")
    for prec, verified in (("fp32", True), ("fp64", True), ("fp32", False)):
        B = FB.BatchSolver([(A, F) for A, F, _ in systems], variant="acifim", precision=prec, memory="device",
                           verified=verified)
        for _ in range(args.warmup):
            tx.zero_()
            B.solve(tb, tx)
        ms = []
        for _ in range(args.steps):
            tx.zero_()
            r = B.solve(tb, tx)
            ms.append(r["summary"]["device_ms"])
        B.close()
        t = max_over_ranks(dist, float(np.mean(ms)))
        key = f"batched_{prec}_factors" + ("" if verified else "_recurrence_test_only")
        out[key] = {
            "solves_per_s": round(args.batch * 1000.0 / t, 2), "ms_per_batch": round(t, 3),
            "max_iter": int(r["iter"].max()), "mean_iter": float(r["iter"].mean()),
            "all_converged": bool((r["info"] == 0).all()), "worst_true_relres": float(r["true_relres"].max()),
            "restart_rounds": r["summary"]["refine_steps"]}
    # (c) plain FP64 GPU solves of the same systems, one after another
    tot, its, trs = 0.0, [], []
    for A, F, bk in systems:
        dA = tuple(torch.from_numpy(a).cuda() for a in A)
        dF = {key: torch.from_numpy(val).cuda() for key, val in F.items()}
        S = FB.Solver(dA, dF, variant="acifim", autotune=False, memory="device")
        tbk = torch.from_numpy(bk).cuda()
        xk = torch.zeros(len(bk), dtype=torch.float64, device="cuda")
        S.solve(tbk, xk, tol=1e-8, nmax=2000)       # warm
        xk.zero_()
        r = S.solve(tbk, xk, tol=1e-8, nmax=2000)
        tot += r["device_ms"]
        its.append(r["iter"])
        trs.append(r["true_relres"])
        S.close()
    tot = max_over_ranks(dist, tot)
    out["sequential_fp64_single_solver"] = {"solves_per_s": round(args.batch * 1000.0 / tot, 2),
                                            "ms_per_batch": round(tot, 3), "max_iter": int(max(its)),
                                            "worst_true_relres": float(max(trs)),
                                            "stop": "the reference's recurrence test"}
    out["ranks"] = world
    out["shard_of_rank0"] = [int(lo), int(hi)] if rank == 0 else None
    out["speedup_batched_fp32_vs_sequential_fp64"] = round(
        out["batched_fp32_factors"]["solves_per_s"] / out["sequential_fp64_single_solver"]["solves_per_s"], 2)
    return out


def run_multi_rhs(args, rank=0, world=1, dist=None):
    """Random nonsymmetric n = 4,000,000 system with Zipf(2.0) row lengths (mean 16, cap 512),
    uniform columns plus the diagonal, off-diagonals U(-1,1), diagonal 1.1 x the absolute row
    sum; 32 right-hand sides N(0,1). Factors: AFIIM eps 0.1 (the example driver's other
    parameters) from the library's construction (the reference's afiim bit for bit; sequential
    in the rows, about two minutes at 4M on one host core), stored FP32 for the block solve;
    --mrhs-factors pdfiim uses the library's PDFIIM eps 0.1 (1,1,1), warpsize 32 instead
    (seconds). AFIIM loop, tol 1e-8, FP64-verified. Compared with the same 32 right-hand sides
    solved one after another by the FP64 single-system solver.

    With N ranks the right-hand sides are sharded: each rank holds the matrix and factors
    and solves a contiguous share of the 32 columns as one block (no exchange on the data
    path); the rates divide all 32 by the max-over-ranks time."""
    import torch
    import fiim_b200 as FB
    n, k = args.mrhs_n, 32
    lo, hi = FB.shard_by_nnz([1] * k, world, rank)
    kr = hi - lo
    t0 = time.perf_counter()
    scale = FB.zipf_scale(n, sample=min(n, 200000))
    A = FB.gen_zipf(n, scale)
    if args.mrhs_factors == "afiim":
        F = FB.afiim_build(A, 0.1)
        fdesc = "AFIIM eps 0.1, library construction (the reference's afiim bit for bit)"
    else:
        F = FB.pdfiim_build(A, 0.1, 1, 1, 1, 32, "I", "B")
        fdesc = "PDFIIM eps 0.1 (1,1,1) warpsize 32, library construction"
    B = (np.stack([FB.rand_normal(n, SEED + 100 + j) for j in range(lo, hi)], axis=1).copy() if kr > 0
         else np.zeros((n, 0)))
    setup = time.perf_counter() - t0
    dev = torch.device("cuda", torch.cuda.current_device())
    tA = tuple(torch.from_numpy(a).to(dev) for a in A)
    tF = {q: torch.from_numpy(v).to(dev) for q, v in F.items()}
    tB = torch.from_numpy(B).to(dev)
    tX = torch.zeros_like(tB)
    out = {"n": n, "nnz": int(A[0][-1]), "rhs": k, "zipf_scale": round(scale, 4), "tol": 1e-8, "loop": "AFIIM",
           "factors": fdesc, "factor_nnz": int(len(F["Gv"]) + len(F["Hv"])), "setup_s": round(setup, 1)}
    t, its_b, conv, worst, rounds = 0.0, 0, True, 0.0, 0
    if kr > 0:
        S = FB.BlockSolver(tA, tF, kr, variant="afiim", precision="fp32", memory="device", verified=True)
        for _ in range(max(1, args.warmup // 2)):
            tX.zero_()
            S.solve(tB, tX)
        ms = []
        for _ in range(max(2, args.steps // 2)):
            tX.zero_()
            r = S.solve(tB, tX)
            ms.append(r["summary"]["device_ms"])
        S.close()
        t = float(np.mean(ms))
        its_b, conv, worst = int(r["iter"].max()), bool((r["info"] == 0).all()), float(r["true_relres"].max())
        rounds = r["summary"]["refine_steps"]
    t = max_over_ranks(dist, t)
    out["block_fp32_factors"] = {"rhs_solves_per_s": round(k * 1000.0 / t, 2), "ms_per_block_solve": round(t, 2),
                                 "max_iter": its_b, "all_converged": conv, "worst_true_relres": worst,
                                 "verified": "FP64 true residual of every right-hand side below tol",
                                 "restart_rounds": rounds}
    tot, its, trs = 0.0, [0], []
    if kr > 0:
        S1 = FB.Solver(tA, tF, variant="afiim", memory="device")
        tx = torch.zeros(n, dtype=torch.float64, device=dev)
        tb = tB[:, 0].contiguous()
        S1.solve(tb, tx)
        for j in range(kr):
            tb = tB[:, j].contiguous()
            tx.zero_()
            r1 = S1.solve(tb, tx)
            tot += r1["device_ms"]
            its.append(r1["iter"])
            trs.append(r1["true_relres"])
        S1.close()
    tot = max_over_ranks(dist, tot)
    out["sequential_fp64_single_rhs"] = {"rhs_solves_per_s": round(k * 1000.0 / tot, 2), "ms_for_32": round(tot, 2),
                                         "max_iter": int(max(its)), "worst_true_relres": float(max(trs or [0.0])),
                                         "stop": "the reference's recurrence test"}
    out["ranks"] = world
    out["rhs_of_rank0"] = [int(lo), int(hi)] if rank == 0 else None
    out["speedup_block_vs_sequential_fp64"] = round(out["block_fp32_factors"]["rhs_solves_per_s"] /
                                                    out["sequential_fp64_single_rhs"]["rhs_solves_per_s"], 2)
    return out


def run_ours(args):
    import torch
    import fiim_b200 as FB
    rank, ws, dist = dist_init("nccl")
    dev = torch.device("cuda", torch.cuda.current_device() if ws > 1 else 0)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    A, b = workload(args.size)
    n, nnz = len(b), int(A[0][-1])
    F = FB.pdfiim_build(A, **PDFIIM_PARAMS)
    t_setup = time.perf_counter() - t0

    # ---- value: device-resident inputs, handle API
    tA = tuple(torch.from_numpy(a).to(dev) for a in A)
    tF = {k: torch.from_numpy(v).to(dev) for k, v in F.items()}
    tb = torch.from_numpy(b).to(dev)
    tx = torch.zeros(n, dtype=torch.float64, device=dev)
    S = FB.Solver(tA, tF, variant="pdfiim", memory="device")
    for _ in range(args.warmup):
        tx.zero_()
        r = S.solve(tb, tx, tol=1e-8, nmax=1200)
    torch.cuda.synchronize()
    barrier(dist)
    results = []
    with Clocks(dev.index) as clk:
        torch.cuda.synchronize()
        barrier(dist)
        w0 = time.perf_counter()
        for _ in range(args.steps):
            tx.zero_()
            results.append(S.solve(tb, tx, tol=1e-8, nmax=1200))
        torch.cuda.synchronize()
        barrier(dist)
        wall = time.perf_counter() - w0
    dev_ms = sum(r["device_ms"] for r in results)
    dev_ms_max = max_over_ranks(dist, dev_ms)
    iters = [r["iter"] for r in results]
    assert all(r["info"] == 0 for r in results), results[0]
    x_fp64 = tx.cpu().numpy()
    value = args.steps * ws / (dev_ms_max / 1000.0)
    it_bytes = S.iteration_bytes()
    hbm_gbs = sum(iters) * it_bytes / (dev_ms / 1000.0) / 1e9
    launches = sum(r["launches"] for r in results)

    # ---- roofline of the dominant kernel (H's SpMV, two launches per iteration). Headline:
    # the body's launches in order with a CUDA event between consecutive ones (each launch
    # as it follows the previous one in the solve), less the events' own cost per launch
    # (the same body timed without them). Beside it: each launch replayed alone, where part
    # of its matrix is still in L2 from the previous replay.
    peak, peak_kind = peaks()
    ktimes = S.kernel_times(reps=20)
    seq, body_ms = S.kernel_times(reps=20, in_sequence=True)
    ev_cost = max(0.0, (sum(m for _, m, _ in seq) - body_ms) / len(seq))
    h_seq = [m for k, m, _ in seq if k == "H_spmv_scale"]
    h_bytes = next(by for k, _, by in seq if k == "H_spmv_scale")
    h_ms = sum(h_seq) / len(h_seq) - ev_cost
    achieved = h_bytes / (h_ms / 1000.0) / 1e9
    h_alone = next(m for k, m, _ in ktimes if k == "H_spmv_scale")
    # The bytes H's product reads in the form it is served in (the formula above counts 4-byte
    # column indices and row offsets; the sliced-diagonal form reads neither), and the
    # iteration's bytes on the same count.
    form_names = {0: "CSR stream", 1: "CSR stream (bulk copies)", 2: "CSR stream (warp blocks)", 3: "sliced-diagonal"}
    nvb = 8.0 * n
    h_form = S.matrix_bytes(2) + 3 * nvb
    it_form = 2 * sum(S.matrix_bytes(w) for w in range(3)) + 32 * nvb
    roofline = {"bound": "hbm", "kernel": "H_spmv_scale", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": args.ncu_traffic, "algorithmic_bytes_per_launch": h_bytes, "launch_ms": round(h_ms, 5),
                "method": "in body order, CUDA events between launches, less the events' cost per launch",
                "event_cost_ms_per_launch": round(ev_cost, 5), "body_ms": round(body_ms, 5),
                "alone": {"launch_ms": round(h_alone, 5), "achieved": round(h_bytes / (h_alone / 1000) / 1e9, 1),
                          "frac": round(h_bytes / (h_alone / 1000) / 1e9 / peak, 4)},
                "per_kernel": [{"kernel": k, "ms": round(m, 5), "gbs": round(by / (m / 1000) / 1e9, 1)}
                               for k, m, by in ktimes],
                "per_kernel_in_sequence": [{"kernel": k, "ms": round(m, 5)} for k, m, _ in seq],
                "form": form_names.get(S.spmv_shape(2)[1], "?"),
                "bytes_note": ("achieved/frac use the survey's formula S(M) = 12 nnz + 4 (n + 1), which counts "
                               "4-byte column indices and row offsets; the sliced-diagonal form reads neither, "
                               "so frac can exceed 1: frac_on_form_bytes and traffic give what it reads"),
                "form_bytes_per_launch": h_form,
                "achieved_on_form_bytes": round(h_form / (h_ms / 1000) / 1e9, 1),
                "frac_on_form_bytes": round(h_form / (h_ms / 1000) / 1e9 / peak, 4),
                "iteration_form_bytes": it_form,
                "hbm_frac_on_form_bytes": round(sum(iters) * it_form / (dev_ms / 1000.0) / 1e9 / peak, 4)}
    # FP64 to the mixed leg's target (1e-10), the reference x for its error
    x_ref10 = None
    if not args.no_mixed:
        tx.zero_()
        r10 = S.solve(tb, tx, tol=1e-10, nmax=1200)
        x_ref10 = tx.clone()
        fp64_10 = {"iter": r10["iter"], "ms": r10["device_ms"], "true_relres": r10["true_relres"]}
    S.close()

    # ---- mixed precision: FP32 BiCGSTAB with FP64 residual replacement (and FP64 refinement)
    mixed, mixed_x = None, {}
    if not args.no_mixed:
        mixed = {"fp64_to_1e-10": fp64_10}
        fp64_8 = dev_ms / args.steps
        # the default form (reliable updates, delta 0.01), and the restarted refinement beside it
        for prec, mtol, rel in (("fp32", 1e-10, None), ("bf16", 1e-10, None), ("fp32", 1e-8, None),
                                ("bf16", 1e-8, None), ("fp32", 1e-8, 0.0)):
            M = FB.Solver(tA, tF, variant="pdfiim", memory="device", precision=prec, inner_tol=1e-5, reliable=rel)
            for _ in range(args.warmup):
                tx.zero_()
                M.solve(tb, tx, tol=mtol, nmax=5000)
            torch.cuda.synchronize()
            rr = []
            for _ in range(args.steps):
                tx.zero_()
                rr.append(M.solve(tb, tx, tol=mtol, nmax=5000))
            ms = sum(q["device_ms"] for q in rr) / len(rr)
            err = float(torch.linalg.norm(tx - x_ref10) / torch.linalg.norm(x_ref10))
            same = fp64_10["ms"] if mtol == 1e-10 else fp64_8
            key = f"{prec}_to_{mtol:g}" + ("_refinement" if rel == 0.0 else "")
            mixed_x[key] = tx.cpu().numpy()
            form = ({"form": "iterative refinement (restarted inner BiCGSTAB)", "inner_tol": 1e-5}
                    if rel == 0.0 else {"form": "reliable updates (FP64 residual replacement)", "delta": 0.01})
            mixed[key] = {
                "solves_per_s": round(1000.0 / ms, 4), "ms_per_solve": round(ms, 4), "tol": mtol, **form,
                "refine_steps": rr[-1]["refine_steps"], "inner_iterations": rr[-1]["iter"],
                "true_relres": rr[-1]["true_relres"], "info": rr[-1]["info"],
                "rel_err_vs_fp64_1e-10_solution": err, "speedup_vs_fp64_same_tol": round(same / ms, 3),
                "a_inner": "FP32 copy of A", "factors": prec.upper(), "d_inv": "FP32"}
            M.close()

    # ---- e2e: reference-facing C-ABI call with pinned host arrays
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, A, F, b, n, ws, dist)

    # ---- batched uneven systems (many small solves in one launch)
    batched = None
    if not args.no_batch:
        batched = run_batched(args, rank, ws, dist)

    # ---- multi-RHS block solve (32 right-hand sides of one n = 4M system)
    multi_rhs = None
    if not args.no_mrhs:
        multi_rhs = run_multi_rhs(args, rank, ws, dist)

    # ---- the small plain case (config 0), latency-bound
    small = None
    if rank == 0 and ws == 1 and not args.no_small:
        small = run_small(args, dev)

    # ---- row-partitioned solve of the one system (headline with --partition rows)
    part = None
    if args.partition == "rows" or (ws == 1 and not args.no_dist):
        part = run_partitioned(args, A, F, b, rank, ws, dist, dev)

    # ---- CPU baseline (rank 0, N = 1): full solves by the reference's own EPBiCGSTAB with its
    # own pdfiim factors; its solutions also give the GPU solutions' distance from the
    # reference's (FP64 to 1e-8, and the mixed legs against its solution to 1e-10).
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cs = CpuSolves(A, b)
        cs.step()                                   # warm-up
        secs, its = [], []
        for _ in range(args.cpu_solves):
            s_, it_, info_, x_ref = cs.step()
            secs.append(s_)
            its.append(it_)
        if cs.kind == "reference":
            its_full, tot = its[-1], sum(secs)
        else:
            its_full = int(np.median(iters))
            tot = sum(s_ * its_full / max(it_, 1) for s_, it_ in zip(secs, its))
        cpu = {"value": len(secs) / tot, "unit": "solves/s", "cores": cs.threads, "kind": cs.kind,
               "sample": cs.describe(len(secs), its_full, sum(secs)), "iterations": its_full}
        if cs.kind == "reference":
            nx = np.linalg.norm(x_ref)
            cpu["gpu_vs_reference"] = {"iterations": [iters[-1], its_full],
                                       "x_rel_diff": float(np.linalg.norm(x_fp64 - x_ref) / nx)}
            if mixed_x:
                x10, _, it10, _, _ = cs.sys.run(b, tol=1e-10, nmax=1200)
                n10 = np.linalg.norm(x10)
                cpu["gpu_vs_reference"]["reference_iterations_to_1e-10"] = it10
                for key, xm in mixed_x.items():
                    mixed[key]["rel_err_vs_reference_fp64_1e-10_solution"] = float(np.linalg.norm(xm - x10) / n10)
        cs.close()

    if rank == 0:
        headline, scaling, par, ms_step = value, "weak", f"replicas x{ws}", dev_ms_max / args.steps
        replicas = None
        if args.partition == "rows":
            replicas = {"value": round(value, 4), "unit": "solves/s", "e2e": e2e}
            headline, scaling, par, ms_step = part["value"], "strong", f"rows x{ws}", part["ms_per_solve"]
            e2e = part["e2e"]
            launches = part["launches_per_solve_per_rank"] * args.steps
        line = {"metric": METRIC, "value": round(headline, 4), "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True,
                "scaling": scaling, "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config(args.size, nnz), "iterations": iters[0], "parallelism": par,
                "setup_s": round(t_setup, 2),
                "hbm_gbs": round(hbm_gbs, 1), "hbm_frac": round(hbm_gbs / peak, 4),
                "iteration_bytes": it_bytes, "true_relres": results[-1]["true_relres"],
                "resval": results[-1]["resval"], "wall_ms_per_step": round(1000 * wall / args.steps, 4),
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "mixed": mixed, "batched": batched, "multi_rhs": multi_rhs,
                "partitioned": part, "replicas": replicas, "small_system": small,
                "gpu_launches": launches,
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=128, help="grid side of the 3D convection-diffusion system")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end C-ABI leg")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-systems leg")
    ap.add_argument("--batch", type=int, default=256, help="systems in the batched leg")
    ap.add_argument("--no-mrhs", action="store_true", help="skip the multi-RHS leg")
    ap.add_argument("--mrhs-n", type=int, default=4000000, help="rows of the multi-RHS system")
    ap.add_argument("--mrhs-factors", default="afiim", choices=["afiim", "pdfiim"],
                    help="factors of the multi-RHS system: AFIIM eps 0.1 (the named config; about two minutes "
                         "to build at 4M) or PDFIIM (seconds)")
    ap.add_argument("--partition", default="replicas", choices=["replicas", "rows"],
                    help="N > 1: replicas of the system per rank (weak scaling, default) or one system in "
                         "row blocks over the ranks (strong scaling)")
    ap.add_argument("--no-dist", action="store_true", help="skip the row-partitioned leg at N = 1")
    ap.add_argument("--no-small", action="store_true", help="skip the small plain case (Poisson 128^2)")
    ap.add_argument("--cpu-solves", type=int, default=3, help="timed full solves of the CPU baseline leg")
    # DRAM bytes per launch of the dominant kernel (H's SpMV) from an ncu capture of the
    # 128^3 workload (dram__bytes_read.sum + dram__bytes_write.sum, mean of three H launches:
    # 0.817 x its algorithmic bytes, the column stream being stored as 16-bit offsets).
    ap.add_argument("--ncu-traffic", type=float, default=220.0e6,
                    help="dram bytes per launch of the dominant kernel from an ncu capture")
    ap.add_argument("--dry-run", action="store_true",
                    help="no GPU: check the rank launcher and max-over-ranks timing over gloo (solves nothing)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        return run_reference(args)
    ws_env = os.environ.get("WORLD_SIZE")
    if ws_env is None and args.gpus > 1:
        return launch_ranks(args)
    if ws_env is not None and int(ws_env) != args.gpus:
        print(f"error: --gpus {args.gpus} but WORLD_SIZE={ws_env}: no result", file=sys.stderr)
        return 2
    return run_dry(args) if args.dry_run else run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
