"""Matrix Market input (the reference's matrix_market_istream,
io/matrix_market.hpp:44-214): the library's reader on files of every
supported kind written here, against CSR built independently in the test;
where the MTL4 tree is available, against the reference's own reader on the
reference's test matrices (bitwise CSR, same accept / refuse decisions)."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT
from mtl4_b200 import _lib
from mtl4_b200 import problems as P
from mtl4_b200.mtl import read_matrix_market


def write_mm(path, header, size_line, lines, comments=("% written by the test",)):
    with open(path, "w") as f:
        f.write(header + "\n")
        for c in comments:
            f.write(c + "\n")
        f.write(size_line + "\n")
        for ln in lines:
            f.write(ln + "\n")


def csr_of(n_rows, n_cols, entries):
    """entries: {(r, c): v} -> (row_ptr, col, val) sorted by row then column."""
    keys = sorted(entries)
    rp = np.zeros(n_rows + 1, np.int64)
    for r, _ in keys:
        rp[r + 1] += 1
    return np.cumsum(rp), np.array([c for _, c in keys], np.int32), np.array([entries[k] for k in keys])


def check_equal(A, n_rows, n_cols, entries):
    rp, ci, v = csr_of(n_rows, n_cols, entries)
    assert (A.n_rows, A.n_cols) == (n_rows, n_cols)
    assert np.array_equal(A.row_ptr, rp) and np.array_equal(A.col, ci) and np.array_equal(A.val, v)


def test_general_real_with_duplicates_and_comments(tmp_path):
    f = tmp_path / "g.mtx"
    write_mm(f, "%%MatrixMarket matrix coordinate real general", "3 4 5",
             ["3 4 -1.5e-3", "1 1 2.0", "2 3 0.0", "1 1 7.25", "3 1 1e300"], comments=("%a", "% b", "%"))
    # a later entry at the same position replaces the earlier one
    check_equal(read_matrix_market(f), 3, 4, {(2, 3): -1.5e-3, (0, 0): 7.25, (1, 2): 0.0, (2, 0): 1e300})


@pytest.mark.parametrize("sym,mirror", [("symmetric", 1.0), ("skew-symmetric", -1.0), ("hermitian", 1.0),
                                        ("SYMMETRIC", 1.0)])
def test_symmetric_kinds_are_mirrored(tmp_path, sym, mirror):
    f = tmp_path / "s.mtx"
    write_mm(f, f"%%MatrixMarket matrix coordinate real {sym}", "3 3 4", ["1 1 4", "2 1 -1", "3 2 0.5", "3 3 2"])
    check_equal(read_matrix_market(f), 3, 3,
                {(0, 0): 4.0, (1, 0): -1.0, (0, 1): -1.0 * mirror, (2, 1): 0.5, (1, 2): 0.5 * mirror, (2, 2): 2.0})


def test_pattern_entries_are_zero_and_integers_convert(tmp_path):
    f = tmp_path / "p.mtx"
    write_mm(f, "%%MatrixMarket matrix coordinate pattern general", "2 2 2", ["1 2", "2 1"])
    check_equal(read_matrix_market(f), 2, 2, {(0, 1): 0.0, (1, 0): 0.0})
    g = tmp_path / "i.mtx"
    write_mm(g, "%%MatrixMarket matrix coordinate integer symmetric", "2 2 2", ["1 1 -3", "2 1 9007199254740993"])
    check_equal(read_matrix_market(g), 2, 2, {(0, 0): -3.0, (1, 0): 9007199254740992.0, (0, 1): 9007199254740992.0})


def test_array_format_is_column_major(tmp_path):
    f = tmp_path / "a.mtx"
    write_mm(f, "%%MatrixMarket matrix array real general", "2 3", ["1", "2", "0", "4", "5", "6"])
    check_equal(read_matrix_market(f), 2, 3, {(0, 0): 1.0, (1, 0): 2.0, (0, 1): 0.0, (1, 1): 4.0, (0, 2): 5.0,
                                              (1, 2): 6.0})


def test_input_that_runs_out_stops_the_entries(tmp_path):
    f = tmp_path / "short.mtx"
    write_mm(f, "%%MatrixMarket matrix coordinate real general", "3 3 5", ["1 1 1", "2 2 2"])
    check_equal(read_matrix_market(f), 3, 3, {(0, 0): 1.0, (1, 1): 2.0})


def test_laplacian_round_trip(tmp_path):
    A = P.laplacian_2d(17)
    f = tmp_path / "lap.mtx"
    lines = []
    for i in range(A.n_rows):
        for e in range(A.row_ptr[i], A.row_ptr[i + 1]):
            if A.col[e] <= i:   # lower triangle, symmetric storage
                lines.append(f"{i + 1} {A.col[e] + 1} {float(A.val[e])!r}")
    write_mm(f, "%%MatrixMarket matrix coordinate real symmetric", f"{A.n_rows} {A.n_cols} {len(lines)}", lines)
    B = read_matrix_market(f)
    assert np.array_equal(B.row_ptr, A.row_ptr) and np.array_equal(B.col, A.col) and np.array_equal(B.val, A.val)


@pytest.mark.parametrize("header,size,lines,exc", [
    ("%%MatrixMarket matrix coordinate complex general", "2 2 1", ["1 1 1 0"], _lib.runtime_error),
    ("%%MatrixMarket vector coordinate real general", "2 2 1", ["1 1 1"], _lib.runtime_error),
    ("%%NotMarket matrix coordinate real general", "2 2 1", ["1 1 1"], _lib.runtime_error),
    ("%%MatrixMarket matrix coordinate double general", "2 2 1", ["1 1 1"], _lib.runtime_error),
    ("%%MatrixMarket matrix coordinate real general", "2 2 1", ["3 1 1"], _lib.runtime_error),
])
def test_malformed_files_are_refused(tmp_path, header, size, lines, exc):
    f = tmp_path / "bad.mtx"
    write_mm(f, header, size, lines)
    with pytest.raises(exc):
        read_matrix_market(f)


def test_missing_file_is_file_not_found(tmp_path):
    with pytest.raises(_lib.file_not_found):
        read_matrix_market(tmp_path / "File_not_exist_test.mtx")


# ---------------------------------------------------------------- reference reader
def reference_tree():
    tree = os.environ.get("MTL4_REFERENCE_TREE", "")
    if not tree:
        tree = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "print-ref"], capture_output=True,
                              text=True).stdout.strip()
    return Path(tree) if tree and Path(tree).is_dir() else None


@pytest.mark.ref
def test_reader_matches_reference_on_its_test_matrices(need_ref):
    tree = reference_tree()
    if tree is None:
        pytest.skip("MTL4 tree not available")
    files = sorted((tree / "libs" / "numeric" / "mtl" / "test" / "matrix_market").glob("*.mtx"))
    assert len(files) >= 6
    compared = 0
    for f in files:
        st, ref = need_ref.ref_matrix_market(f)
        try:
            A = read_matrix_market(f)
        except _lib.MtlError:
            A = None
        if st != 0:
            # the reference refuses it (complex values into a real matrix,
            # files without the header): so does the library
            assert A is None, f.name
            continue
        nr, nc, rp, ci, v = ref
        assert (A.n_rows, A.n_cols) == (nr, nc), f.name
        assert np.array_equal(A.row_ptr, rp) and np.array_equal(A.col, ci), f.name
        assert np.array_equal(A.val, v), f.name
        compared += 1
    assert compared >= 4
