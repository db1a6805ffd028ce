"""Seeded generators for the sparse systems the solvers are measured on.

All matrices are returned as CSR triplets ``(row_ptr int64[n+1], col int32[nnz],
val float64[nnz])`` with columns sorted inside every row, which is the layout
``mtl::compressed2D`` keeps (boost/numeric/mtl/matrix/compressed2D.hpp:259) and
the one the triangular solves require (operation/lower_trisolve.hpp:105).

Row numbering of grid problems is lexicographic with the first coordinate
fastest, as ``laplacian_setup`` numbers a 2D grid (row = i * n + j,
boost/numeric/mtl/matrix/laplacian_setup.hpp:26-41).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class CSR:
    n_rows: int
    n_cols: int
    row_ptr: np.ndarray  # int64[n_rows + 1]
    col: np.ndarray      # int32[nnz]
    val: np.ndarray      # float64[nnz]

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """y = A x in FP64 with a per-row sequential sum (numpy reduceat)."""
        prod = self.val * x[self.col]
        y = np.zeros(self.n_rows, dtype=np.float64)
        nz = np.diff(self.row_ptr) > 0
        if prod.size:
            y[nz] = np.add.reduceat(prod, self.row_ptr[:-1][nz])
        return y

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.row_ptr), shape=(self.n_rows, self.n_cols))


def _from_coo(n: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray) -> CSR:
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=row_ptr[1:])
    return CSR(n, n, row_ptr, cols.astype(np.int32), vals.astype(np.float64))


def laplacian_2d(m: int, n: int | None = None) -> CSR:
    """5-point Laplacian on an m x n grid, Dirichlet: 4 on the diagonal and -1
    on the neighbours (laplacian_setup.hpp:26-41)."""
    n = m if n is None else n
    N = m * n
    idx = np.arange(N, dtype=np.int64)
    i, j = idx // n, idx % n
    rows = [idx]
    cols = [idx]
    vals = [np.full(N, 4.0)]
    for mask, off in ((j < n - 1, 1), (i < m - 1, n), (j > 0, -1), (i > 0, -n)):
        rows.append(idx[mask])
        cols.append(idx[mask] + off)
        vals.append(np.full(int(mask.sum()), -1.0))
    return _from_coo(N, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def _grid_neighbours_3d(m: int):
    N = m ** 3
    idx = np.arange(N, dtype=np.int64)
    x = idx % m
    y = (idx // m) % m
    z = idx // (m * m)
    coords = (x, y, z)
    strides = (1, m, m * m)
    return N, idx, coords, strides


def convdiff_3d(m: int, beta=(0.5, 0.3, 0.2), h: float | None = None) -> CSR:
    """7-point -Laplace(u) + beta . grad(u) on an m^3 grid, centred
    differences, Dirichlet, h = 1/(m+1).  Diagonal 6/h^2; neighbour in
    direction d: -1/h^2 - beta_d/(2h) below, -1/h^2 + beta_d/(2h) above.
    Nonsymmetric whenever beta != 0."""
    h = 1.0 / (m + 1) if h is None else h
    N, idx, coords, strides = _grid_neighbours_3d(m)
    rows, cols, vals = [idx], [idx], [np.full(N, 6.0 / (h * h))]
    for d in range(3):
        c, s = coords[d], strides[d]
        lo, hi = c > 0, c < m - 1
        rows += [idx[lo], idx[hi]]
        cols += [idx[lo] - s, idx[hi] + s]
        vals += [np.full(int(lo.sum()), -1.0 / (h * h) - beta[d] / (2 * h)),
                 np.full(int(hi.sum()), -1.0 / (h * h) + beta[d] / (2 * h))]
    return _from_coo(N, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def _face_diffusion(shape, kappa: np.ndarray, beta=None, h: float = 1.0) -> CSR:
    """Cell-centred diffusion with per-cell coefficients kappa (flattened,
    first axis fastest).  Face coefficient = arithmetic mean of the two cells;
    a boundary face takes the cell's own coefficient (Dirichlet) and only adds
    to the diagonal.  Optional centred convection beta (per axis)."""
    dims = len(shape)
    N = int(np.prod(shape))
    idx = np.arange(N, dtype=np.int64)
    coords = []
    stride = 1
    strides = []
    for d in range(dims):
        coords.append((idx // stride) % shape[d])
        strides.append(stride)
        stride *= shape[d]
    diag = np.zeros(N)
    rows, cols, vals = [], [], []
    for d in range(dims):
        c, s = coords[d], strides[d]
        for side in (-1, 1):
            inside = (c > 0) if side < 0 else (c < shape[d] - 1)
            nb = idx + side * s
            face = np.where(inside, 0.5 * (kappa + kappa[np.where(inside, nb, idx)]), kappa)
            diag += face / (h * h)
            conv = 0.0 if beta is None else side * beta[d] / (2 * h)
            rows.append(idx[inside])
            cols.append(nb[inside])
            vals.append(-face[inside] / (h * h) + conv)
    rows.append(idx)
    cols.append(idx)
    vals.append(diag)
    return _from_coo(N, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def vardiff_3d(m, sigma: float = 1.0, seed: int = 3, beta=None) -> CSR:
    """SPD 7-point diffusion on an m^3 grid (or an (nx, ny, nz) grid, x
    fastest) with log-normal cell coefficients (kappa ~ exp(N(0, sigma^2)),
    seeded), face value = arithmetic mean of the two cells, Dirichlet.  With
    beta, adds centred convection (nonsymmetric)."""
    shape = tuple(m) if isinstance(m, (tuple, list)) else (m, m, m)
    rng = np.random.default_rng(seed)
    kappa = np.exp(sigma * rng.standard_normal(int(np.prod(shape))))
    return _face_diffusion(shape, kappa, beta)


def vardiff_2d(m, sigma: float = 1.0, seed: int = 3, beta=None) -> CSR:
    """2D 5-point counterpart of :func:`vardiff_3d` on an m x m (or (nx, ny)) grid."""
    shape = tuple(m) if isinstance(m, (tuple, list)) else (m, m)
    rng = np.random.default_rng(seed)
    kappa = np.exp(sigma * rng.standard_normal(int(np.prod(shape))))
    return _face_diffusion(shape, kappa, beta)


# Continuous Pareto (density ~ x^-alpha, alpha = 2.1) floored and clipped to
# [1, 4096].  x_min = 1.55 gives a mean row length of ~9.5, i.e. ~40M entries
# on 4,194,304 rows; x_min = 1 would give ~6.3 (~26M entries).
POWERLAW_XMIN = 1.55


def powerlaw_csr(n: int = 4 * 2 ** 20, alpha: float = 2.1, lo: int = 1, hi: int = 4096,
                 seed: int = 2, x_min: float = POWERLAW_XMIN) -> CSR:
    """Irregular square CSR: row lengths floor(Pareto(alpha, x_min)) clipped to
    [lo, hi]; columns uniform on [0, n) without duplicates, sorted; values
    N(0, 1).  Seeded."""
    rng = np.random.default_rng(seed)
    u = rng.random(n)
    lengths = np.floor(x_min * (1.0 - u) ** (-1.0 / (alpha - 1.0)))
    lengths = np.clip(lengths, lo, min(hi, n)).astype(np.int64)
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lengths, out=row_ptr[1:])
    nnz = int(row_ptr[-1])
    rows = np.repeat(np.arange(n, dtype=np.int64), lengths)
    cols = rng.integers(0, n, size=nnz, dtype=np.int64)
    # Resample duplicates inside a row until every row's columns are distinct.
    for _ in range(64):
        key = rows * n + cols
        order = np.argsort(key, kind="stable")
        ks = key[order]
        dup = np.zeros(nnz, dtype=bool)
        dup[order[1:][ks[1:] == ks[:-1]]] = True
        ndup = int(dup.sum())
        if ndup == 0:
            break
        cols[dup] = rng.integers(0, n, size=ndup, dtype=np.int64)
    key = rows * n + cols
    order = np.argsort(key, kind="stable")
    cols = cols[order]
    vals = rng.standard_normal(nnz)
    return CSR(n, n, row_ptr, cols.astype(np.int32), vals)


def rhs_from_solution(A: CSR, seed: int):
    """x_true ~ U(-1, 1) (seeded) and b = A x_true in FP64."""
    rng = np.random.default_rng(seed)
    x_true = rng.uniform(-1.0, 1.0, A.n_cols)
    return x_true, A.matvec(x_true)


def random_rhs(n: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)


# ---------------------------------------------------------------- configs

def config1():
    """Plain FP64 CG + diagonal on the 256x256 5-point Laplacian; b = A x_true,
    x_true ~ U(-1,1) seed 0; rtol 1e-8, max 2000 iterations."""
    A = laplacian_2d(256)
    x_true, b = rhs_from_solution(A, 0)
    return A, b, x_true


def config2_solve(m: int = 128):
    """BiCGSTAB + ILU(0) on the 3D convection-diffusion operator, m^3 grid,
    beta = (0.5, 0.3, 0.2), h = 1/(m+1); b = A x_true, seed 1; rtol 1e-8."""
    A = convdiff_3d(m)
    x_true, b = rhs_from_solution(A, 1)
    return A, b, x_true


def config2_spmv(n: int = 4 * 2 ** 20):
    """Standalone SpMV operand: the power-law irregular CSR (seed 2)."""
    return powerlaw_csr(n, seed=2)


def config3a(m: int = 2048):
    A = laplacian_2d(m)
    x_true, b = rhs_from_solution(A, 3)
    return A, b, x_true


def config3b(m: int = 160):
    A = vardiff_3d(m, sigma=1.0, seed=3)
    x_true, b = rhs_from_solution(A, 3)
    return A, b, x_true


@dataclass
class SystemSpec:
    """One system of a batch or a request stream."""
    dims: int          # 2 or 3
    m: int             # grid edge (n = m^dims unknowns)
    sigma: float
    seed: int
    pc: str            # "diagonal" | "ic_0" | "ilu_0"
    solver: str        # "cg" | "bicgstab"
    beta: tuple | None = None

    @property
    def n(self) -> int:
        return self.m ** self.dims

    def build(self) -> CSR:
        if self.dims == 2:
            return vardiff_2d(self.m, self.sigma, self.seed, self.beta)
        return vardiff_3d(self.m, self.sigma, self.seed, self.beta)


def batch_specs(count: int = 1024, n_lo: float = 1e3, n_hi: float = 2.56e5, seed: int = 4,
                sigma: float = 0.5):
    """Uneven batch: sizes log-uniform in [n_lo, n_hi] (rounded to a grid),
    half 2D 5-point and half 3D 7-point diffusion, each with its own
    log-normal coefficients; PC diagonal or IC(0) drawn per system."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(n_lo), math.log(n_hi), count))
    specs = []
    for s in range(count):
        dims = 2 if s % 2 == 0 else 3
        m = max(2, int(round(sizes[s] ** (1.0 / dims))))
        pc = "diagonal" if rng.random() < 0.5 else "ic_0"
        specs.append(SystemSpec(dims, m, sigma, int(seed * 1_000_003 + s), pc, "cg"))
    return specs


def request_specs(count: int = 20000, n_lo: float = 4e3, n_hi: float = 2e6, seed: int = 5,
                  sigma: float = 1.0, conv_frac: float = 0.2):
    """Served stream: sizes log-uniform in [n_lo, n_hi], 2D or 3D, log-normal
    coefficients; 20% carry a convection term with |beta| ~ U(0,1) and use
    BiCGSTAB + ILU(0), the rest CG + IC(0)."""
    rng = np.random.default_rng(seed)
    specs = []
    for s in range(count):
        n = math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))
        dims = 2 if rng.random() < 0.5 else 3
        m = max(2, int(round(n ** (1.0 / dims))))
        if rng.random() < conv_frac:
            mag = rng.uniform(0.0, 1.0)
            direction = rng.standard_normal(dims)
            direction /= np.linalg.norm(direction)
            # |beta| on the unit cube, scaled by h = 1/(m+1) into grid units
            beta = tuple(float(v) for v in mag * direction / (m + 1))
            specs.append(SystemSpec(dims, m, sigma, int(seed * 1_000_003 + s), "ilu_0", "bicgstab", beta))
        else:
            specs.append(SystemSpec(dims, m, sigma, int(seed * 1_000_003 + s), "ic_0", "cg"))
    return specs


def poisson_arrivals(count: int, rate: float, seed: int = 5) -> np.ndarray:
    """Open-loop Poisson arrival times (seconds) at `rate` requests/s."""
    rng = np.random.default_rng(seed + 7919)
    return np.cumsum(rng.exponential(1.0 / rate, count))
