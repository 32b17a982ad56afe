"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs here, where the reference tree is present: the reference's own construction
(afiim / pdfiim / acifim) and solve (EPBiCGSTAB / PBiCGSTAB) code, compiled unmodified
against oracle/mkl_shim by `make -C oracle ref`, on one thread. The reference ships
no golden outputs of its own (it has no tests); its only fixture is the HB/sherman2
system in */example/, which is stored here together with what the reference computes
on it. Matrices of the synthetic workloads come from the product's generators (the
reference has none), seeded as the benchmark seeds them.

Usage:  python tests/golden/make_golden.py [--reference /path/to/reference]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "computational-mathematics_b200"))
import pyoracle as O  # noqa: E402
import fiim_b200 as FB  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
SEED = 20261203


def csr(prefix, A):
    return {f"{prefix}i": np.asarray(A[0], np.int32), f"{prefix}j": np.asarray(A[1], np.int32),
            f"{prefix}v": np.asarray(A[2], np.float64)}


def factors(F, with_lu=False):
    keys = ["Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv"] + (["Li", "Lj", "Lv", "Ui", "Uj", "Uv"] if with_lu else [])
    return {k: F[k] for k in keys if F.get(k) is not None}


def probe(A, F, n, sym=False, nr=None):
    """A seeded probe vector with the reference-semantics products the GPU must match."""
    u = FB.rand_normal(n, SEED + 1)
    out = {"u": u, "Au": O.csr_mv(*A, u) if not sym else O.csr_mv_sym_upper(*A, u)}
    out["Mu"] = O.prec_apply(F, u, sym=sym)
    if nr is not None:
        out["MuC"] = O.prec_apply_combined(F, u, nr)
    return out


# Summation orders sampled for the rounding envelope: the dot products and norms split
# into B contiguous blocks (the MKL shim's OpenMP reduction on B threads).
BLOCKS = list(range(1, 49)) + [64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536, 2048, 3072, 4096]


def solved(prefix, variant, A, b, F, tol, nmax, **kw):
    """One-thread reference run (bit-identical to the restatement) plus its rounding envelope:
    the iteration counts the same solve takes when only the summation order of its dot
    products and norms changes. The restatement with B blocks is the reference on B threads
    (checked here for B = 2, 3, 5, 8); the envelope runs the restatement over BLOCKS and
    counts the runs that end with the same info as the one-thread run."""
    O.set_threads(1, variant)
    O.set_dot_blocks(1)
    x, res, it, info = O.ref_solve(variant, A, b, F, tol=tol, nmax=nmax, **kw)
    xr, resr, itr, infor = O.bicgstab(variant, A, b, F, tol=tol, nmax=nmax, **kw)
    assert np.array_equal(x, xr) and res == resr and it == itr and info == infor, "restatement drifted"
    for B in (2, 3, 5, 8):
        O.set_threads(B, variant)
        O.set_dot_blocks(B)
        xa, *ra = O.ref_solve(variant, A, b, F, tol=tol, nmax=nmax, **kw)
        xb, *rb = O.bicgstab(variant, A, b, F, tol=tol, nmax=nmax, **kw)
        assert ra == rb and np.array_equal(xa, xb), f"blocked restatement drifted at B={B}"
    its, spread, infos = [], 0.0, set()
    for B in BLOCKS:
        O.set_dot_blocks(B)
        xt, _, itt, inft = O.bicgstab(variant, A, b, F, tol=tol, nmax=nmax, **kw)
        infos.add(inft)
        if inft != info:
            continue
        its.append(itt)
        spread = max(spread, float(np.linalg.norm(xt - x) / np.linalg.norm(x)))
    O.set_dot_blocks(1)
    O.set_threads(1, variant)
    return {f"{prefix}x": x, f"{prefix}resval": np.float64(res), f"{prefix}iter": np.int32(it),
            f"{prefix}info": np.int32(info), f"{prefix}iter_env": np.array([min(its), max(its)], np.int32),
            f"{prefix}x_spread": np.float64(spread)}, \
        {"resval": res, "iter": it, "info": info, "iter_env": [min(its), max(its)], "x_spread": spread,
         "infos": sorted(infos), "orders": len(BLOCKS), "same_info": len(its)}


def save(name, arrays, meta):
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, meta=np.array(json.dumps(meta)), **arrays)
    print(f"{name}: {os.path.getsize(path) / 1024:.0f} KB  {meta.get('results')}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("FIIM_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference")))
    args = ap.parse_args()
    for pkg in ("afiim", "pdfiim", "acifim"):
        O.set_threads(1, pkg)

    # 1. HB/sherman2, the reference's example system (AFIIM/README:29, ACIFIM/README:31).
    S = O.read_matrix(os.path.join(args.reference, "AFIIM/example/sherman2.mtx"))
    n = len(S[0]) - 1
    bs = O.read_rhs(os.path.join(args.reference, "AFIIM/example/sherman2_rhs1.mtx"), n)
    arrays = {**csr("A", S), "b": bs}
    meta = {"system": "HB/sherman2", "results": {}}
    for tag, dtol in (("afiim9e-6", 9e-6), ("afiim0.1", 0.1)):
        F = O.afiim_build(S, dtol)
        arrays.update({f"{tag}_{k}": v for k, v in factors(F).items()})
        arrays.update({f"{tag}_{k}": v for k, v in probe(S, F, n).items()})
        r, m = solved(f"{tag}_", "afiim", S, bs, F, 1e-8, 500)
        arrays.update(r)
        meta["results"][tag] = m
    Fc, cerr = O.acifim_build(S, 0.01, 0.01)
    assert cerr == 0
    arrays.update({f"acifim_{k}": v for k, v in factors(Fc, True).items()})
    arrays.update({f"acifim_{k}": v for k, v in probe(S, Fc, n, nr=2).items()})
    for mode in "EC":
        r, m = solved(f"acifim{mode}_", "acifim", S, bs, Fc, 1e-8, 2000, mode=mode, nr=2)
        arrays.update(r)
        meta["results"][f"acifim{mode}"] = m
    Fp = O.pdfiim_build(S, 0.01, 2, 2, 1, -1, "I", "B")
    arrays.update({f"pdfiim_{k}": v for k, v in factors(Fp).items()})
    r, m = solved("pdfiim_", "pdfiim", S, bs, Fp, 1e-8, 1200)
    arrays.update(r)
    meta["results"]["pdfiim"] = m
    meta["params"] = {"afiim": "elemPerRowCol 10, growth 5, eta 0, shift 0",
                      "acifim": "dtol1 0.01, dtol2 0.01, elemPerRowCol 30, growth 5, coeff 2, element_limit 200, filtit 30, nr 2",
                      "pdfiim": "ftol 0.01, prefill 2, lfill 2, postfill 1, warpsize -1, 'I', 'B'"}
    save("sherman2", arrays, meta)

    # 2. Poisson 128x128, b = A*1, x0 = 0, AFIIM eps 0.1, tol 1e-8, NMAX 1000 (plain FP64 case).
    A = FB.gen_poisson2d(128)
    b = FB.model_rhs(A)
    F = O.afiim_build(A, 0.1)
    r, m = solved("", "afiim", A, b, F, 1e-8, 1000)
    save("poisson128_afiim", {**csr("A", A), "b": b, **factors(F), **probe(A, F, len(b)), **r},
         {"system": "2D 5-point Poisson 128x128, Dirichlet", "factors": "afiim eps 0.1", "results": m})

    # 3. 3D convection-diffusion 16^3 (the 128^3 workload's stencil), PDFIIM (2,2,1) eps 0.05.
    A = FB.gen_convdiff3d(16, 0.5)
    b = FB.rand_normal(len(A[0]) - 1, SEED)
    F = O.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    r, m = solved("", "pdfiim", A, b, F, 1e-8, 1200)
    save("convdiff16_pdfiim", {**csr("A", A), "b": b, **factors(F), **probe(A, F, len(b)), **r},
         {"system": "3D 7-point upwind convection-diffusion 16^3, cell Peclet 0.5",
          "factors": "pdfiim ftol 0.05 prefill 2 lfill 2 postfill 1 warpsize -1 'I' 'B'", "results": m})

    # 4. 2D convection-diffusion 48^2 with the first batched system's coefficients, ACIFIM (0.1, 0.05).
    _, diff, theta, pe = FB.batch_params(SEED, 0)
    A = FB.gen_convdiff2d(48, diff, theta, pe)
    b = FB.rand_normal(48 * 48, SEED + 2)
    F, cerr = O.acifim_build(A, 0.1, 0.05)
    assert cerr == 0
    arrays = {**csr("A", A), "b": b, **factors(F, True), **probe(A, F, len(b), nr=2)}
    res = {}
    for mode in "EC":
        r, m = solved(f"{mode}_", "acifim", A, b, F, 1e-8, 2000, mode=mode, nr=2)
        arrays.update(r)
        res[mode] = m
    save("convdiff2d48_acifim", arrays,
         {"system": f"2D 5-point upwind convection-diffusion 48^2, diff {diff}, theta {theta}, Peclet {pe}",
          "factors": "acifim dtol1 0.1 dtol2 0.05 (driver defaults otherwise), nr 2", "results": res})

    # 5. PDFIIM symmetric input: Poisson 32x32 stored as its upper triangle (mtype SYMMETRIC);
    #    G from pdfiim on the full matrix; the solver applies z = G (D^{-1} o (G^T r)) as
    #    PDFIIM/src/bicgstab.cpp:189-194 does.
    Af = FB.gen_poisson2d(32)
    F = O.pdfiim_build(Af, 0.05, 2, 2, 1, -1, "I", "B")
    Ai, Aj, Av = Af
    keep = np.concatenate([[0], np.cumsum([np.sum(Aj[Ai[i]:Ai[i + 1]] >= i) for i in range(len(Ai) - 1)])]).astype(np.int32)
    mask = np.concatenate([Aj[Ai[i]:Ai[i + 1]] >= i for i in range(len(Ai) - 1)])
    Au = (keep, Aj[mask].astype(np.int32), Av[mask])
    b = FB.rand_normal(32 * 32, SEED + 3)
    Fs = {k: F[k] for k in ("Gi", "Gj", "Gv", "IDv")}
    r, m = solved("", "pdfiim", Au, b, Fs, 1e-8, 1200, issym=True)
    save("poisson32_sym_pdfiim", {**csr("A", Au), "b": b, **Fs, **probe(Au, Fs, len(b), sym=True), **r},
         {"system": "2D Poisson 32x32, upper triangle, SYMMETRIC", "factors": "pdfiim ftol 0.05 (2,2,1) G only",
          "results": m})


if __name__ == "__main__":
    main()
