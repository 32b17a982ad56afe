"""The reference's example programs relink unchanged against libfiim_b200.so.

AFIIM/example/example.cpp, ACIFIM/example/example.cpp and PDFIIM/example/pdfiim.cpp are
built twice from the reference tree (oracle/Makefile, target `drivers`): as shipped, with
the reference's bicgstab.cpp, and with bicgstab.cpp left out and libfiim_b200.so linked in
its place. Both run here on HB/sherman2, written back to Matrix Market files from the golden
fixture (the reference reader's CSR arrays and right-hand side), with each driver's own
built-in parameters, which are those of the fixture's factors.

CPU: the shipped programs reproduce the fixture (iterations and x bit for bit on one
thread), which pins the file writer and the output parsing below; the relinked programs
take their solver symbols from the library and, with no GPU, stop with its error.
GPU: the relinked programs solve on the B200 and meet the drop-in parity bar of
test_gpu_solve.py (info, iterations within the reference's rounding envelope +-2, x within
10x the reference's own spread).
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

REFBIN = os.path.join(ROOT, "oracle", "_ref")
LIB = os.path.join(ROOT, "computational-mathematics_b200", "libfiim_b200.so")

# program, argv after the two file names, golden prefix of the reference's solve, solver
# symbol the program calls. The parameters are the drivers' command-line ones matching the
# fixture's factors (tests/golden/make_golden.py, sherman2).
CASES = [
    ("afiim_example", ["9e-6"], "afiim9e-6_", "EPBiCGSTAB"),
    ("afiim_example", ["0.1"], "afiim0.1_", "EPBiCGSTAB"),
    ("acifim_example", ["0.01", "0.01", "2", "E"], "acifimE_", "PBiCGSTAB"),
    ("acifim_example", ["0.01", "0.01", "2", "C"], "acifimC_", "PBiCGSTAB"),
    ("pdfiim_example", ["2", "2", "1", "0.01", "-1"], "pdfiim_", "EPBiCGSTAB"),
]
IDS = [f"{c[0]}-{c[2].rstrip('_')}" for c in CASES]


def program(name):
    p = os.path.join(REFBIN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not built (oracle/Makefile `drivers` needs the reference tree)")
    return p


def write_system(g, d):
    """sherman2 as the reference's reader expects it: coordinate real general for A
    (1-based, row by row), array real general for b; %r keeps every double exact."""
    Ai, Aj, Av, b = g["Ai"], g["Aj"], g["Av"], g["b"]
    n = len(Ai) - 1
    a, r = os.path.join(d, "A.mtx"), os.path.join(d, "b.mtx")
    rows = np.repeat(np.arange(n), np.diff(Ai))
    with open(a, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{n} {n} {len(Aj)}\n")
        f.writelines(f"{i + 1} {j + 1} {float(v)!r}\n" for i, j, v in zip(rows, Aj, Av))
    with open(r, "w") as f:
        f.write("%%MatrixMarket matrix array real general\n")
        f.write(f"{n} 1\n")
        f.writelines(f"{float(v)!r}\n" for v in b)
    return a, r


def run(prog, g, d, args, timeout=300):
    a, r = write_system(g, d)
    if not os.access(prog, os.X_OK):
        # a copy of the repository that dropped the mode bits: run a private copy (the
        # library is then found through LD_LIBRARY_PATH instead of the run path)
        local = os.path.join(d, os.path.basename(prog))
        shutil.copyfile(prog, local)
        os.chmod(local, 0o755)
        prog = local
    pkg = os.path.dirname(LIB)
    env = dict(os.environ, OMP_NUM_THREADS="1",
               LD_LIBRARY_PATH=os.pathsep.join(filter(None, [pkg, os.environ.get("LD_LIBRARY_PATH")])))
    return subprocess.run([prog, a, r, *args], cwd=d, capture_output=True, text=True, env=env, timeout=timeout)


def parse(out):
    """(iterations, info) from a driver's output: the solver's own verbose line (AFIIM,
    PDFIIM) or the ACIFIM driver's summary lines."""
    m = re.search(r"Convergence in (\d+) iterations with relative residual", out)
    if m:
        return int(m.group(1)), 0
    it = re.search(r"Iterations to convergence\s*:\s*(-?\d+)", out)
    info = re.search(r"CIFIM-PBiCGSTAB info\s*:\s*(-?\d+)", out)
    assert it and info, out[-2000:]
    return int(it.group(1)), int(info.group(1))


def read_solution(d):
    lines = [ln for ln in open(os.path.join(d, "solution.mtx")) if not ln.startswith("%")]
    n = int(lines[0].split()[0])
    x = np.array([float(v) for v in lines[1:1 + n]])
    assert len(x) == n
    return x


def solver_symbols(path):
    """{solver name: nm type letter} for the BiCGSTAB symbols of an executable."""
    out = subprocess.run(["nm", "-C", path], capture_output=True, text=True, check=True).stdout
    syms = {}
    for ln in out.splitlines():
        m = re.match(r"^\s*[0-9a-f]*\s+([A-Za-z])\s+(\w*BiCGSTAB)\(", ln)
        if m:
            syms[m.group(2)] = m.group(1)
    return syms


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.parametrize("name", ["afiim_example", "acifim_example", "pdfiim_example"])
def test_relinked_program_takes_the_solver_from_the_library(name):
    """The shipped program defines its solver; the relinked one leaves it undefined and the
    dynamic linker resolves it from libfiim_b200.so (its run path, from any copy)."""
    shipped, relinked = program(name), program(name + "_fiim")
    sym = {"acifim_example": "PBiCGSTAB"}.get(name, "EPBiCGSTAB")
    assert solver_symbols(shipped).get(sym) in ("T", "t")   # defined in the program
    assert solver_symbols(relinked).get(sym) == "U"
    ldd = subprocess.run(["ldd", relinked], capture_output=True, text=True).stdout
    line = next(ln for ln in ldd.splitlines() if "libfiim_b200.so" in ln)
    assert "not found" not in line
    assert os.path.realpath(line.split("=>")[1].split("(")[0].strip()) == os.path.realpath(LIB)


@pytest.mark.parametrize("name,args,prefix,sym", CASES, ids=IDS)
def test_shipped_program_reproduces_fixture(golden, tmp_path, name, args, prefix, sym):
    """The reference's own program, on the rewritten files, gives the fixture's iterations
    and x bit for bit: the files and the parsing are the reference's own inputs and outputs."""
    g = golden("sherman2")
    p = run(program(name), g, str(tmp_path), args)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    it, info = parse(p.stdout)
    assert (it, info) == (int(g[prefix + "iter"]), int(g[prefix + "info"]))
    assert np.array_equal(read_solution(str(tmp_path)), g[prefix + "x"])


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
@pytest.mark.parametrize("name,args,prefix,sym", CASES[1:2] + CASES[2:3] + CASES[4:], ids=IDS[1:3] + IDS[4:])
def test_relinked_program_stops_without_gpu(golden, tmp_path, name, args, prefix, sym):
    """With no GPU the relinked program reaches the library's solver, which throws its
    error instead of computing on the CPU; no solution file is written."""
    p = run(program(name + "_fiim"), golden("sherman2"), str(tmp_path), args)
    assert p.returncode != 0
    assert "fiim_b200: no CUDA device visible" in p.stderr
    assert not os.path.exists(tmp_path / "solution.mtx")


@pytest.mark.gpu
@pytest.mark.parametrize("name,args,prefix,sym", CASES, ids=IDS)
def test_relinked_program_solves_on_gpu(golden, tmp_path, name, args, prefix, sym):
    """The unchanged reference program, its solver calls served by the library on the B200,
    meets the drop-in parity bar against the reference's solve of the same system."""
    g = golden("sherman2")
    p = run(program(name + "_fiim"), g, str(tmp_path), args)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    it, info = parse(p.stdout)
    lo, hi = (int(v) for v in g[prefix + "iter_env"])
    x, xr = read_solution(str(tmp_path)), g[prefix + "x"]
    dx = np.linalg.norm(x - xr) / np.linalg.norm(xr)
    print(f"{name} {' '.join(args)}: iter {it} info {info} | ref {int(g[prefix + 'iter'])} "
          f"envelope [{lo},{hi}] | x rel diff {dx:.2e}")
    assert info == int(g[prefix + "info"])
    assert lo - 2 <= it <= hi + 2
    assert dx <= 10 * float(g[prefix + "x_spread"]) + 1e-9
