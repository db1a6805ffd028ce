"""Python mirror of MTL4's iterative solvers (ITL) on the GPU.

Same names and argument meaning as boost/numeric/itl:
  basic_iteration(r0_or_norm, max_iter, rtol, atol)  itl/iteration/basic_iteration.hpp:24-164
  cg(A, x, b, P, iter)                               itl/krylov/cg.hpp:76
  bicgstab(A, x, b, P, iter)                         itl/krylov/bicgstab.hpp:29
  gmres(A, x, b, L, R, iter, restart)                itl/krylov/gmres.hpp:124
  pc.identity / diagonal / ilu_0 / ic_0 (A, value)   itl/pc/*.hpp
  solve(P, x), adjoint_solve(P, x)
The solvers return iter.error_code() as the reference does; BiCGSTAB
breakdown raises unexpected_orthogonality.
"""
from __future__ import annotations

import ctypes as C
import sys
import math

import numpy as np

from . import _lib
from ._lib import check, unexpected_orthogonality  # noqa: F401  (re-exported)
from .mtl import compressed2D, dense_vector, two_norm


class basic_iteration:
    """Termination control.  Constructed from a vector (norm_r0 = ||r0||, e.g.
    b) or from a number (basic_iteration.hpp:31-39)."""

    def __init__(self, r0_or_norm, max_iter: int, rtol: float, atol: float = 0.0):
        if isinstance(r0_or_norm, dense_vector):
            self._norm_r0 = two_norm(r0_or_norm)
        elif isinstance(r0_or_norm, np.ndarray):
            self._norm_r0 = float(np.linalg.norm(r0_or_norm))
        else:
            self._norm_r0 = abs(float(r0_or_norm))
        self.max_iter = int(max_iter)
        self.rtol = float(rtol)
        self._atol = float(atol)
        self.i = 0
        self.error = 0
        self._resid = 0.0
        self.status = _lib.ST_RUNNING
        self.seconds = 0.0
        self.outer = 0
        self.fp64_fallback = False   # refinement finished by a plain FP64 solve

    # reference accessors
    def iterations(self) -> int: return self.i
    def max_iterations(self) -> int: return self.max_iter
    def error_code(self) -> int: return self.error
    def resid(self) -> float: return self._resid
    def relresid(self) -> float: return self._resid / self._norm_r0 if self._norm_r0 else self._resid
    def norm_r0(self) -> float: return self._norm_r0
    def tol(self) -> float: return self.rtol
    def atol(self) -> float: return self._atol
    def is_converged(self) -> bool: return self.status == _lib.ST_CONVERGED and self.error == 0
    def __int__(self) -> int: return self.error

    def _params(self, restart: int = 0) -> _lib.IterParams:
        return _lib.IterParams(self.max_iter, int(restart), self.rtol, self._atol, self._norm_r0)

    def _take(self, r: _lib.IterResult):
        self.i = r.iterations
        self.error = r.error_code
        self._resid = r.resid
        self.status = r.status
        self.seconds = r.seconds
        self.outer = r.outer_iterations
        self.fp64_fallback = bool(r.fp64_fallback)
        if r.norm_r0 > 0 or self._norm_r0 == 0:
            self._norm_r0 = r.norm_r0


class cyclic_iteration(basic_iteration):
    """basic_iteration that prints the residual every `cycle` iterations and
    a summary from error_code(), as the reference's cyclic_iteration
    (itl/iteration/cyclic_iteration.hpp:22-95).  The termination tests run on
    the device; their (iteration, residual) log is replayed through
    finished() after the solve, so the lines are the ones the reference's
    loop prints (C++ stream formatting: 6 significant digits)."""

    wants_log = True

    def __init__(self, r0_or_norm, max_iter: int, rtol: float, atol: float = 0.0, cycle: int = 100, out=None):
        super().__init__(r0_or_norm, max_iter, rtol, atol)
        self.cycle = int(cycle)
        self.last_print = -1
        self.multi_print = False
        self.quiet = False
        self.suppress = False
        self.out = out if out is not None else sys.stdout

    def set_multi_print(self, m: bool):
        self.multi_print = bool(m)

    def set_cycle(self, c: int):
        self.cycle = int(c)

    def finished(self, r: float) -> bool:
        """basic_iteration::finished(r) (basic_iteration.hpp:43-65), then the
        cycle's print-out."""
        self._resid = float(r)
        nr0 = self._norm_r0
        conv = (r <= self._atol) if nr0 == 0 else (r <= self.rtol * nr0 or r <= self._atol)
        done = conv
        if not conv and self.i >= self.max_iter:
            self.error, done = 1, True
        if not self.quiet and self.i % self.cycle == 0 and (self.multi_print or self.i != self.last_print):
            self.out.write(f"iteration {self.i}: resid {_g(self._resid)}\n")
            self.last_print = self.i
        return done

    def error_code(self) -> int:
        if not self.suppress:
            it = max(self.i, 1)
            self.out.write(f"finished! error code = {self.error}\n{self.i} iterations\n"
                           f"{_g(self._resid)} is actual final residual. \n"
                           f"{_g(self.relresid())} is actual relative tolerance achieved. \n"
                           f"Relative tol: {_g(self.rtol)}  Absolute tol: {_g(self._atol)}\n"
                           f"Convergence:  {_g(self.relresid() ** (1.0 / it))}\n")
        return self.error

    def _replay(self, log, r: _lib.IterResult):
        for k in range(len(log) // 2):
            self.i = int(log[2 * k])
            self.finished(float(log[2 * k + 1]))
        self.i = max(self.i, r.iterations)


class noisy_iteration(cyclic_iteration):
    """cyclic_iteration printing every iteration (itl/iteration/noisy_iteration.hpp:22-35)."""

    def __init__(self, r0_or_norm, max_iter: int, rtol: float, atol: float = 0.0, out=None):
        super().__init__(r0_or_norm, max_iter, rtol, atol, 1, out)


def _g(v: float) -> str:
    """A double as std::ostream prints it by default (%g, 6 digits)."""
    return "%g" % v


class pc:
    """Preconditioners (itl::pc)."""

    class _base:
        kind = _lib.PC_IDENTITY

        def __init__(self, A: compressed2D, value=np.float64, tune: bool = True):
            self.A = A
            self.ctx = A.ctx
            self.value = np.dtype(value)
            if tune and self.kind in (_lib.PC_ILU0, _lib.PC_IC0) and self.ctx.autotune is not None:
                from . import autotune, mtl
                name = "ilu_0" if self.kind == _lib.PC_ILU0 else "ic_0"
                mtl.tuned(A, ("pc", name, self.value.name),
                          lambda ctx, Ad, cache: autotune.tune_pc(ctx, Ad, name, self.value, cache))
            h = C.c_void_p()
            st = _lib.F64 if self.value == np.float64 else _lib.F32
            check(self.ctx._L.mtlg_pc_create(self.ctx.h, A.h, self.kind, st, C.byref(h)), type(self).__name__)
            self.h = h

        def levels(self):
            a, b = C.c_int(), C.c_int()
            check(self.ctx._L.mtlg_pc_levels(self.h, C.byref(a), C.byref(b)), "levels")
            return a.value, b.value

        def sweep_plan(self, dtype=np.float64) -> dict:
            """Launch plan of the sweeps for vectors of `dtype` under the
            context's tuning: "kernel" is "grid" (grid-stencil factors: tiles,
            steps per warp unit), "chunked" (chunk rows and count, staging) or
            "flat" (level order, all other fields zero)."""
            out = (C.c_int * 8)()
            dt = _lib.F32 if np.dtype(dtype) == np.float32 else _lib.F64
            check(self.ctx._L.mtlg_pc_sweep_plan(self.ctx.h, self.h, dt, out), "sweep_plan")
            v = list(out)
            if v[1] == 0 and v[2] > 0:
                keys = ("chunk_rows", "chunks", "resident", "smem", "threads", "entries", "tiles", "steps")
                return dict(zip(keys, v), kernel="grid")
            keys = ("chunk_rows", "chunks", "resident", "smem", "threads", "entries", "seg_rows", "seg_ents")
            return dict(zip(keys, v), kernel="chunked" if v[1] > 0 else "flat")

        def factor(self, which: str):
            """Stored factor ('L' or 'U') as (row_ptr, col, val) host arrays."""
            w = 0 if which == "L" else 1
            nnz = C.c_int64()
            check(self.ctx._L.mtlg_pc_factor(self.h, w, C.byref(nnz), None, None, None), "factor")
            n = self.A.num_rows()
            rp = np.zeros(n + 1, np.int64)
            ci = np.zeros(max(nnz.value, 1), np.int32)
            v = np.zeros(max(nnz.value, 1), np.float64)
            check(self.ctx._L.mtlg_pc_factor(self.h, w, C.byref(nnz), C.c_void_p(rp.ctypes.data),
                                             C.c_void_p(ci.ctypes.data), C.c_void_p(v.ctypes.data)), "factor")
            return rp, ci[:nnz.value], v[:nnz.value]

        def get_L(self):
            return self.factor("L")

        def get_U(self):
            return self.factor("U")

        def __del__(self):
            try:
                if getattr(self, "h", None) and self.ctx.h:
                    self.ctx._L.mtlg_pc_destroy(self.h)
            except Exception:
                pass

    class identity(_base):
        kind = _lib.PC_IDENTITY

    class diagonal(_base):
        kind = _lib.PC_DIAGONAL

    class ilu_0(_base):
        kind = _lib.PC_ILU0

    class ic_0(_base):
        kind = _lib.PC_IC0


def solve(P: pc._base, x: dense_vector, y: dense_vector | None = None) -> dense_vector:
    """y = solve(P, x)."""
    y = y or dense_vector(x.n, x.dtype, x.ctx)
    check(P.ctx._L.mtlg_pc_apply(P.ctx.h, P.h, x.h, y.h), "solve")
    return y


def adjoint_solve(P: pc._base, x: dense_vector, y: dense_vector | None = None) -> dense_vector:
    y = y or dense_vector(x.n, x.dtype, x.ctx)
    check(P.ctx._L.mtlg_pc_adjoint_apply(P.ctx.h, P.h, x.h, y.h), "adjoint_solve")
    return y


def _solve(kind, A, x, b, L, R, it: basic_iteration, restart=0, tune=True) -> int:
    from .mtl import poisson2D_dirichlet
    if isinstance(A, poisson2D_dirichlet):
        return _solve_poisson(kind, A, x, b, it, restart)
    if tune and A.ctx.autotune is not None:
        _tune_vec(A)
    res = _lib.IterResult()
    params = it._params(restart)
    logged = getattr(it, "wants_log", False)
    if logged:
        A.ctx.ensure_residual_log(2 * it.max_iter + 8)
    st = A.ctx._L.mtlg_solve(A.ctx.h, kind, A.h, L.h if L is not None else None, R.h if R is not None else None,
                             x.h, b.h, C.byref(params), C.byref(res))
    if logged:
        log = A.ctx.residual_log()
        norm_r0 = it._norm_r0
        it._take(res)
        if log is not None and len(log):
            it._norm_r0 = norm_r0 if res.norm_r0 <= 0 else res.norm_r0
            err, resid = it.error, it._resid
            it._replay(log, res)
            it.error, it._resid = err, resid
    else:
        it._take(res)
    check(st, _SOLVER_NAME.get(kind, "solve"))
    return it.error_code()


_SOLVER_NAME = {_lib.CG: "cg", _lib.BICGSTAB: "bicgstab", _lib.GMRES: "gmres", _lib.BICG: "bicg", _lib.CGS: "cgs",
                _lib.TFQMR: "tfqmr", _lib.QMR: "qmr", _lib.BICGSTAB_2: "bicgstab_2",
                _lib.BICGSTAB_ELL: "bicgstab_ell", _lib.IDR_S: "idr_s"}


def _tune_vec(A):
    from . import autotune, mtl
    mtl.tuned(A, "vec", lambda ctx, Ad, cache: autotune.tune_vec(ctx, Ad, np.float64, cache))


def _solve_poisson(kind, A, x, b, it: basic_iteration, restart=0) -> int:
    """Solves on the matrix-free poisson2D_dirichlet operator (host-driven,
    no preconditioning)."""
    res = _lib.IterResult()
    params = it._params(restart)
    st = A.ctx._L.mtlg_poisson2d_solve(A.ctx.h, kind, A.m, A.n, x.h, b.h, C.byref(params), C.byref(res))
    it._take(res)
    check(st, "poisson2D solve")
    return it.error_code()


def cg(A, x, b, P, it: basic_iteration, tune: bool = True) -> int:
    return _solve(_lib.CG, A, x, b, P, None, it, tune=tune)


def bicgstab(A, x, b, P, it: basic_iteration) -> int:
    return _solve(_lib.BICGSTAB, A, x, b, P, None, it)


def gmres(A, x, b, L, R, it: basic_iteration, restart: int) -> int:
    return _solve(_lib.GMRES, A, x, b, L, R, it, restart)


# Host-driven bodies on device vectors (itl/krylov/*.hpp), FP64.
def bicg(A, x, b, P, it: basic_iteration) -> int:
    return _solve(_lib.BICG, A, x, b, P, None, it)


def cgs(A, x, b, P, it: basic_iteration) -> int:
    return _solve(_lib.CGS, A, x, b, P, None, it)


def tfqmr(A, x, b, L, R, it: basic_iteration) -> int:
    return _solve(_lib.TFQMR, A, x, b, L, R, it)


def qmr(A, x, b, L, R, it: basic_iteration) -> int:
    return _solve(_lib.QMR, A, x, b, L, R, it)


def bicgstab_2(A, x, b, P, it: basic_iteration) -> int:
    return _solve(_lib.BICGSTAB_2, A, x, b, P, None, it)


def bicgstab_ell(A, x, b, L, R, it: basic_iteration, ell: int) -> int:
    return _solve(_lib.BICGSTAB_ELL, A, x, b, L, R, it, ell)


def idr_s(A, x, b, L, R, it: basic_iteration, s: int) -> int:
    return _solve(_lib.IDR_S, A, x, b, L, R, it, s)


def refine(solver: str, A: compressed2D, x: dense_vector, b: dense_vector, P, rtol: float = 1e-8,
           inner_rtol: float = 1e-4, max_outer: int = 20, max_inner: int = 2000) -> basic_iteration:
    """FP64 iterative refinement around an FP32 inner solve (no reference
    counterpart).  x, b: FP64; P: preconditioner stored in FP32.  When an
    outer step fails to halve the FP64 residual (an operator too
    ill-conditioned for FP32) or the inner solve breaks down, the system is
    finished by a plain FP64 solve (it.fp64_fallback is then True)."""
    kind = {"cg": _lib.CG, "bicgstab": _lib.BICGSTAB}[solver]
    if A.ctx.autotune is not None:
        _tune_vec(A)
    rp = _lib.RefineParams(int(max_outer), int(max_inner), 0, 0, float(rtol), float(inner_rtol))
    res = _lib.IterResult()
    st = A.ctx._L.mtlg_refine_solve(A.ctx.h, kind, A.h, P.h if P is not None else None, x.h, b.h, C.byref(rp),
                                    C.byref(res))
    it = basic_iteration(res.norm_r0 if res.norm_r0 else 1.0, max_inner, rtol)
    it._take(res)
    check(st, "refine")
    return it
