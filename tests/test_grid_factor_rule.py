"""The rule the grid factorization rests on, checked on CPU against the
oracle's ILU(0) and IC(0) factors (no GPU): on a 5- or 7-point grid stencil
in natural order a row's pivot needs only its earlier neighbours' pivots --
ILU(0) (boost/numeric/itl/pc/ilu_0.hpp:45-82, sides of at least 3): for each
earlier neighbour k by ascending column, l = a_ik / u_kk (rounded product
with the inverse pivot) and u_ii = fma(-l, a_ki, u_ii), every other entry
unchanged; IC(0) (ic_0.hpp:124-186): d = a_ki / sqrt(u_kk) and u_ii -= d * d
with rounded products.  The rule holds for sides of 2 as well (the column
an earlier neighbour shares with the row by index never exists on both
sides of the grid boundary); the library still leaves such ILU(0) grids to
the level-scheduled kernel."""
import math
from fractions import Fraction

import numpy as np
import pytest

from mtl4_b200 import problems as P
from oracle import oracle as O


def fma(a, b, c):
    # correctly rounded a * b + c (exact rational, then one rounding)
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def entry(A, r, c):
    lo, hi = A.row_ptr[r], A.row_ptr[r + 1]
    k = np.searchsorted(A.col[lo:hi], c)
    return float(A.val[lo + k]) if k < hi - lo and A.col[lo + k] == c else None


def grid_pivots(A, shape, kind):
    nx, ny, nz = shape
    n = A.n_rows
    inv = np.zeros(n)
    for r in range(n):
        i, j, k = r % nx, (r // nx) % ny, r // (nx * ny)
        nbrs = [r - nx * ny] if k > 0 else []
        nbrs += [r - nx] if j > 0 else []
        nbrs += [r - 1] if i > 0 else []
        d = entry(A, r, r)
        for q in nbrs:   # ascending column
            if kind == "ilu_0":
                l = entry(A, r, q) * inv[q]
                d = fma(-l, entry(A, q, r), d)
            else:
                t = entry(A, q, r) * inv[q]
                d = d - t * t
        inv[r] = 1.0 / d if kind == "ilu_0" else 1.0 / math.sqrt(d)
    return inv


def diagonal_of(rp, ci, v):
    n = rp.size - 1
    out = np.zeros(n)
    for r in range(n):
        cols = ci[rp[r]:rp[r + 1]]
        out[r] = v[rp[r] + int(np.nonzero(cols == r)[0][0])]
    return out


GRIDS = [
    (P.vardiff_3d((6, 5, 4), sigma=1.0, seed=3, beta=(0.3, 0.2, 0.1)), (6, 5, 4)),
    (P.vardiff_2d((9, 7), sigma=1.0, seed=4, beta=(0.2, 0.1)), (9, 7, 1)),
    (P.convdiff_3d(5), (5, 5, 5)),
]


@pytest.mark.parametrize("A,shape", GRIDS)
@pytest.mark.parametrize("kind", ["ilu_0", "ic_0"])
def test_grid_pivots_equal_the_oracle_factorization(A, shape, kind):
    if kind == "ic_0":
        A = P.vardiff_3d(shape, sigma=1.0, seed=3) if shape[2] > 1 else P.vardiff_2d(shape[:2], sigma=1.0, seed=4)
    inv = grid_pivots(A, shape, kind)
    U = O.port_factor(A, kind, "U")
    assert np.array_equal(diagonal_of(*U), inv)
    if kind == "ilu_0":
        # L entries are a_ik times the inverse pivot of k, U's off-diagonal
        # entries are A's: nothing but the pivots changes
        rp, ci, v = O.port_factor(A, kind, "L")
        for r in range(A.n_rows):
            for e in range(rp[r], rp[r + 1]):
                assert v[e] == entry(A, r, int(ci[e])) * inv[ci[e]]
        rp, ci, v = U
        for r in range(A.n_rows):
            for e in range(rp[r], rp[r + 1]):
                if ci[e] != r:
                    assert v[e] == entry(A, r, int(ci[e]))


@pytest.mark.parametrize("shape", [(5, 2, 4), (2, 6, 3), (2, 2, 5), (2, 7, 1)])
def test_rule_holds_with_sides_of_two(shape):
    A = P.vardiff_3d(shape, sigma=1.0, seed=5, beta=(0.3, 0.2, 0.1)) if shape[2] > 1 else \
        P.vardiff_2d(shape[:2], sigma=1.0, seed=5, beta=(0.3, 0.2))
    inv = grid_pivots(A, shape, "ilu_0")
    rp, ci, v = O.port_factor(A, "ilu_0", "U")
    assert np.array_equal(diagonal_of(rp, ci, v), inv)
    assert all(v[e] == entry(A, r, int(ci[e])) for r in range(A.n_rows) for e in range(rp[r], rp[r + 1])
               if ci[e] != r)
