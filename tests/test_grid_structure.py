"""Grid-stencil detection of factor patterns (host logic, no GPU): the
preconditioners whose factor pattern is a 5- or 7-point grid stencil in
natural order get the grid sweep and factorization; every other pattern
keeps the chunked and flat kernels.  Checked on grids of several shapes
(lower and upper parts, the entry orders the kernel runs) and on patterns
that must be refused."""
import ctypes as C

import numpy as np
import pytest

from mtl4_b200 import problems as P


def structure(A, lower=True):
    from mtl4_b200 import _lib
    L = _lib.load()
    rp = np.ascontiguousarray(A.row_ptr, dtype=np.int64)
    ci = np.ascontiguousarray(A.col, dtype=np.int32)
    out = (C.c_int * 8)()
    assert L.mtlg_grid_structure(A.n_rows, rp.ctypes.data, ci.ctypes.data, 1 if lower else 0, out) == 0
    return list(out)


@pytest.mark.parametrize("A,shape", [
    (P.laplacian_2d(31), (31, 31, 1)),
    (P.vardiff_2d((50, 300), sigma=1.0, seed=8, beta=(0.2, 0.1)), (50, 300, 1)),
    (P.convdiff_3d(20), (20, 20, 20)),
    (P.vardiff_3d((33, 40, 13), sigma=1.0, seed=4), (33, 40, 13)),
    (P.vardiff_3d((7, 70, 9), sigma=0.5, seed=6), (7, 70, 9)),
])
def test_grids_are_detected(A, shape):
    ns = 2 if shape[2] == 1 else 3
    lo, up = structure(A, True), structure(A, False)
    # rows stored by ascending column: L reads its farthest neighbour first,
    # U its nearest
    assert lo[:6] == [*shape, ns, 1, 1]
    assert up[:6] == [*shape, ns, 2, 1]


def _csr(n, rows, cols):
    vals = np.ones(len(rows))
    return P._from_coo(n, np.asarray(rows), np.asarray(cols), vals)


def test_non_grid_patterns_are_refused():
    m = 12
    n = m * m
    # 9-point stencil: four lower offsets
    rows, cols = [], []
    for r in range(n):
        i, j = r % m, r // m
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                if 0 <= i + di < m and 0 <= j + dj < m:
                    rows.append(r); cols.append(r + di + m * dj)
    assert structure(_csr(n, rows, cols))[0] == 0
    # 5-point with x wrapping around (periodic): row i = 0 reads row r - 1
    rows, cols = [], []
    for r in range(n):
        rows.append(r); cols.append(r)
        if r > 0: rows.append(r); cols.append(r - 1)
        if r >= m: rows.append(r); cols.append(r - m)
    assert structure(_csr(n, rows, cols))[0] == 0
    # a 2D grid with one extra entry
    A = P.laplacian_2d(m)
    rows = list(np.repeat(np.arange(n), np.diff(A.row_ptr))) + [n - 1]
    cols = list(A.col) + [0]
    assert structure(_csr(n, rows, cols))[0] == 0
    # a grid under a symmetric permutation
    perm = np.random.default_rng(1).permutation(n)
    inv = np.argsort(perm)
    r0 = np.repeat(np.arange(n), np.diff(A.row_ptr))
    assert structure(_csr(n, inv[r0], inv[A.col]))[0] == 0
    # tridiagonal (a single chain: no second direction)
    rows = [r for r in range(n) for _ in (0, 1)][1:]
    cols = [c for r in range(n) for c in (r - 1, r)][1:]
    assert structure(_csr(n, rows, cols))[0] == 0


def test_pattern_without_entries_is_a_grid_of_independent_rows():
    n = 1000
    out = structure(_csr(n, list(range(n)), list(range(n))))
    assert out[:6] == [256, 4, 1, 0, 0, 0]
