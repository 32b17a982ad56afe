"""Host input/output (no GPU): the Matrix Market readers against the reference's own reader
(compiled from its sources into the oracle), the right-hand-side reader, and the binary
factor file's round trip and damage checks."""
import os

import numpy as np
import pytest

import fiim_b200 as FB
import pyoracle as O
from conftest import load_golden

REFERENCE = O.REFERENCE   # the reference tree, where present
REF_SHERMAN2 = os.path.join(REFERENCE, "AFIIM/example/sherman2.mtx")
REF_SHERMAN2_RHS = os.path.join(REFERENCE, "AFIIM/example/sherman2_rhs1.mtx")


def write_mtx(path, n, rows, cols, vals, symmetry="general"):
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real {symmetry}\n% written by the test\n")
        f.write(f"{n} {n} {len(rows)}\n")
        for i, j, v in zip(rows, cols, vals):
            f.write(f"{i + 1} {j + 1} {float(v)!r}\n")


def random_entries(n, m, seed, lower=False, dups=0):
    rng = np.random.default_rng(seed)
    rows, cols = rng.integers(0, n, m), rng.integers(0, n, m)
    if lower:
        rows, cols = np.maximum(rows, cols), np.minimum(rows, cols)
    rows = np.concatenate([rows, np.arange(n), rows[:dups]])
    cols = np.concatenate([cols, np.arange(n), cols[:dups]])
    vals = rng.standard_normal(len(rows)) * 10.0 ** rng.integers(-8, 8, len(rows))
    order = rng.permutation(len(rows))
    return rows[order], cols[order], vals[order]


@pytest.mark.skipif(not os.path.exists(REF_SHERMAN2), reason="reference example files not present")
def test_sherman2_matches_golden_reference_csr():
    g = load_golden("sherman2")
    (Ai, Aj, Av), sym = FB.read_mtx(REF_SHERMAN2)
    assert not sym
    assert np.array_equal(Ai, g["Ai"]) and np.array_equal(Aj, g["Aj"]) and np.array_equal(Av, g["Av"])
    b = FB.read_rhs(REF_SHERMAN2_RHS)
    assert np.array_equal(b, g["b"])


@pytest.mark.parametrize("symmetry,dups", [("general", 0), ("general", 40), ("symmetric", 0), ("symmetric", 25)])
def test_reader_matches_reference_reader(tmp_path, symmetry, dups):
    """Shuffled entries, repeated entries and symmetric storage: the same arrays, bit for
    bit, as the reference's read_coeff_matrix (AFIIM/src/rw_matrix.cpp:62-216)."""
    if not O.have_ref("afiim"):
        pytest.skip("reference library not built")
    n = 300
    rows, cols, vals = random_entries(n, 2500, 11 + dups, lower=(symmetry == "symmetric"), dups=dups)
    path = str(tmp_path / "m.mtx")
    write_mtx(path, n, rows, cols, vals, symmetry)
    (Ai, Aj, Av), sym = FB.read_mtx(path)
    Ri, Rj, Rv = O.read_matrix(path)
    assert not sym
    assert np.array_equal(Ai, Ri) and np.array_equal(Aj, Rj) and np.array_equal(Av, Rv)


# Files of at least 65,536 entries are parsed in pieces on all host threads; these cases
# hold 150,000 and more, so they take that path.
LARGE_N, LARGE_M = 20000, 150000


@pytest.mark.parametrize("symmetry,dups", [("general", 0), ("general", 3000), ("symmetric", 0),
                                           ("symmetric", 2000)])
def test_large_reader_matches_reference_reader(tmp_path, symmetry, dups):
    """The piecewise parse of a large file gives the reference reader's arrays bit for bit."""
    if not O.have_ref("afiim"):
        pytest.skip("reference library not built")
    rows, cols, vals = random_entries(LARGE_N, LARGE_M, 7 + dups, lower=(symmetry == "symmetric"), dups=dups)
    path = str(tmp_path / "m.mtx")
    write_mtx(path, LARGE_N, rows, cols, vals, symmetry)
    (Ai, Aj, Av), _ = FB.read_mtx(path)
    Ri, Rj, Rv = O.read_matrix(path)
    assert np.array_equal(Ai, Ri) and np.array_equal(Aj, Rj) and np.array_equal(Av, Rv)
    if symmetry == "symmetric":
        (Ui, Uj, Uv), sym = FB.read_mtx(path, form="pdfiim")
        assert sym and len(Uj) == len(rows)
        r_of = np.repeat(np.arange(LARGE_N), np.diff(Ui))
        assert (Uj >= r_of).all()


def _layout(rows, cols, vals, how):
    """Entry text laid out otherwise than one entry per line; the reference reads tokens
    with fscanf, whatever the line breaks."""
    ent = [f"{i + 1} {j + 1} {float(v)!r}" for i, j, v in zip(rows, cols, vals)]
    if how == "several_per_line":
        return "\n".join("  ".join(ent[k:k + 3]) for k in range(0, len(ent), 3)) + "\n"
    if how == "broken_entries":
        return "".join(e.replace(" ", "\n", 1) + "\n" if k % 7 == 0 else e + "\n" for k, e in enumerate(ent))
    if how == "blank_lines_crlf":
        return "".join(e + ("\r\n\r\n" if k % 5 == 0 else "\r\n") for k, e in enumerate(ent))
    if how == "signs_and_exponents":
        return "".join(f"{i + 1}\t{j + 1}\t{'+' if v >= 0 else ''}{float(v):.17e}\n"
                       for i, j, v in zip(rows, cols, vals))
    if how == "trailing_text":
        return "\n".join(ent) + "\n% not an entry\nend of file\n"
    raise ValueError(how)


@pytest.mark.parametrize("how", ["several_per_line", "broken_entries", "blank_lines_crlf", "signs_and_exponents",
                                 "trailing_text"])
def test_large_reader_layouts_match_reference_reader(tmp_path, how):
    """Line layouts that a piece cannot split on (entries broken across lines, text after
    the entries) and ones it can (several entries per line, blank lines, CRLF, signs):
    either way the arrays are the reference reader's."""
    if not O.have_ref("afiim"):
        pytest.skip("reference library not built")
    rows, cols, vals = random_entries(LARGE_N, LARGE_M, 3)
    path = str(tmp_path / "m.mtx")
    with open(path, "w", newline="") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{LARGE_N} {LARGE_N} {len(rows)}\n")
        f.write(_layout(rows, cols, vals, how))
    (Ai, Aj, Av), _ = FB.read_mtx(path)
    Ri, Rj, Rv = O.read_matrix(path)
    assert np.array_equal(Ai, Ri) and np.array_equal(Aj, Rj) and np.array_equal(Av, Rv)


def test_large_reader_errors_name_the_entry(tmp_path):
    """A bad entry in a large file is reported with its position, as for a small one; a file
    with fewer entries than its size line declares is rejected."""
    rows, cols, vals = random_entries(LARGE_N, LARGE_M, 4)
    rows = rows.copy()
    rows[100000] = LARGE_N + 5
    path = str(tmp_path / "m.mtx")
    write_mtx(path, LARGE_N, rows, cols, vals)
    with pytest.raises(FB.FiimError, match=rf"entry 100001 \({LARGE_N + 6}, \d+\) is outside"):
        FB.read_mtx(path)
    rows[100000] = 0
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{LARGE_N} {LARGE_N} {len(rows) + 10}\n")
        f.writelines(f"{i + 1} {j + 1} {float(v)!r}\n" for i, j, v in zip(rows, cols, vals))
    with pytest.raises(FB.FiimError, match=rf"entry {len(rows) + 1} is malformed"):
        FB.read_mtx(path)


def test_pdfiim_form_keeps_the_upper_triangle(tmp_path):
    """PDFIIM's reader (PDFIIM/src/rw_matrix.cpp:104-150) reads a symmetric file as its mirror
    image: the lower-stored entries become the upper triangle, flagged symmetric. Its
    symmetric expansion equals the AFIIM form's matrix."""
    import scipy.sparse as sp
    n = 200
    rows, cols, vals = random_entries(n, 1500, 5, lower=True)
    keep = np.unique(np.stack([rows, cols], 1), axis=0, return_index=True)[1]
    rows, cols, vals = rows[keep], cols[keep], vals[keep]
    path = str(tmp_path / "s.mtx")
    write_mtx(path, n, rows, cols, vals, "symmetric")
    (Ui, Uj, Uv), sym = FB.read_mtx(path, form="pdfiim")
    assert sym
    r_of = np.repeat(np.arange(n), np.diff(Ui))
    assert (Uj >= r_of).all()
    for i in range(n):
        assert (np.diff(Uj[Ui[i]:Ui[i + 1]]) > 0).all()
    U = sp.csr_matrix((Uv, Uj, Ui), shape=(n, n))
    full = (U + sp.triu(U, 1).T).tocsr()
    full.sort_indices()
    (Ai, Aj, Av), _ = FB.read_mtx(path, form="afiim")
    assert np.array_equal(full.indptr, Ai) and np.array_equal(full.indices, Aj) and np.array_equal(full.data, Av)


@pytest.mark.parametrize("banner", ["%%MatrixMarket matrix coordinate complex general",
                                    "%%MatrixMarket matrix coordinate pattern general",
                                    "%%MatrixMarket matrix coordinate integer general",
                                    "%%MatrixMarket matrix coordinate real skew-symmetric",
                                    "%%MatrixMarket matrix array real general"])
def test_reader_rejects_unsupported_types(tmp_path, banner):
    path = str(tmp_path / "bad.mtx")
    with open(path, "w") as f:
        f.write(banner + "\n2 2 1\n1 1 1.0\n")
    with pytest.raises(FB.FiimError):
        FB.read_mtx(path)


def test_reader_rejects_non_square_and_missing(tmp_path):
    path = str(tmp_path / "rect.mtx")
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n2 3 1\n1 1 1.0\n")
    with pytest.raises(FB.FiimError, match="not square"):
        FB.read_mtx(path)
    with pytest.raises(FB.FiimError, match="does not exist"):
        FB.read_mtx(str(tmp_path / "none.mtx"))


def test_rhs_reader_matches_reference(tmp_path):
    if not O.have_ref("afiim"):
        pytest.skip("reference library not built")
    b = np.random.default_rng(2).standard_normal(77) * 1e3
    path = str(tmp_path / "b.mtx")
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix array real general\n% rhs\n77 1\n")
        f.writelines(f"{float(v)!r}\n" for v in b)
    got = FB.read_rhs(path)
    assert np.array_equal(got, O.read_rhs(path, 77)) and np.array_equal(got, b)


def test_factor_file_round_trip_and_damage(tmp_path):
    A = FB.gen_convdiff3d(10, 0.5)
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1, -1, "I", "B")
    path = str(tmp_path / "f.bin")
    FB.factors_save(path, F)
    G = FB.factors_load(path)
    for k in F:
        assert np.array_equal(F[k], G[k]), k
    raw = bytearray(open(path, "rb").read())
    raw[100] ^= 0x40
    bad = str(tmp_path / "bad.bin")
    open(bad, "wb").write(bytes(raw))
    with pytest.raises(FB.FiimError, match="checksum"):
        FB.factors_load(bad)
    open(bad, "wb").write(bytes(raw[:len(raw) // 2]))
    with pytest.raises(FB.FiimError):
        FB.factors_load(bad)
    open(bad, "wb").write(b"NOTAFILE" + bytes(64))
    with pytest.raises(FB.FiimError, match="not a factor file"):
        FB.factors_load(bad)
