"""Test infrastructure only: Python access to the two CPU oracles.

* ``ref``  -- oracle/_ref/libmtlref.so: MTL4's own headers, unchanged, built by
  oracle/Makefile (the reference itself; also the timed CPU baseline).
* ``port`` -- oracle/_build/libmtloracle.so: the project's CPU restatement
  (oracle/mtl_oracle.cpp), pinned against ``ref`` and the reference tests'
  known-answer vectors.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product never does.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libmtlref.so"
REF_OMP_LIB = HERE / "_ref" / "libmtlref_omp.so"
PORT_LIB = HERE / "_build" / "libmtloracle.so"

PC_KIND = {"identity": 0, "diagonal": 1, "ilu_0": 2, "ic_0": 3}
SOLVER = {"cg": 0, "bicgstab": 1, "gmres": 2, "bicg": 3, "cgs": 4, "tfqmr": 5, "qmr": 6, "bicgstab_2": 7,
          "bicgstab_ell": 8, "idr_s": 9}


class RefResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("error", C.c_int), ("resid", C.c_double), ("relresid", C.c_double),
                ("setup_s", C.c_double), ("solve_s", C.c_double), ("outer", C.c_int), ("pad", C.c_int)]


class PortResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("error", C.c_int), ("resid", C.c_double), ("relresid", C.c_double),
                ("outer", C.c_int), ("pad", C.c_int)]


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


_REF = {}
_PORT = None


def ref_available(omp: bool = False) -> bool:
    return (REF_OMP_LIB if omp else REF_LIB).exists()


def ref_lib(omp: bool = False) -> C.CDLL:
    key = bool(omp)
    if key not in _REF:
        L = C.CDLL(str(REF_OMP_LIB if omp else REF_LIB))
        VP = C.c_void_p
        L.mtlref_csr_create.restype = VP
        L.mtlref_csr_create.argtypes = [C.c_int64, C.c_int64, C.c_int64, VP, VP, VP]
        L.mtlref_csr_destroy.argtypes = [VP]
        L.mtlref_openmp_threads.restype = C.c_int
        L.mtlref_spmv.argtypes = [VP, VP, VP, C.c_int]
        L.mtlref_spmv_f32.argtypes = [VP, VP, VP, C.c_int]
        L.mtlref_spmv_timed.restype = C.c_double
        L.mtlref_spmv_timed.argtypes = [VP, VP, VP, C.c_int]
        L.mtlref_dot.restype = C.c_double
        L.mtlref_dot.argtypes = [C.c_int64, VP, VP]
        L.mtlref_two_norm.restype = C.c_double
        L.mtlref_two_norm.argtypes = [C.c_int64, VP]
        L.mtlref_pc_apply.argtypes = [VP, C.c_int, C.c_int, VP, VP]
        L.mtlref_pc_apply_f32.argtypes = [VP, C.c_int, VP, VP]
        L.mtlref_pc_adjoint_apply.argtypes = [VP, C.c_int, C.c_int, VP, VP]
        PI = C.POINTER(C.c_int64)
        L.mtlref_pc_factors.argtypes = [VP, C.c_int, PI, VP, VP, VP, PI, VP, VP, VP]
        L.mtlref_solve.argtypes = [VP, C.c_int, C.c_int, C.c_int, VP, VP, C.c_int, C.c_double, C.c_double, C.c_int,
                                   C.POINTER(RefResult)]
        L.mtlref_solve_f32.argtypes = [VP, C.c_int, C.c_int, VP, VP, C.c_int, C.c_double, C.c_double, C.c_int,
                                       C.POINTER(RefResult)]
        L.mtlref_refine_solve.argtypes = [VP, C.c_int, C.c_int, VP, VP, C.c_int, C.c_int, C.c_double, C.c_double,
                                          C.c_int, C.POINTER(RefResult)]
        L.mtlref_laplacian_setup.argtypes = [C.c_int, C.c_int, PI, VP, VP, VP]
        L.mtlref_solve_krylov.argtypes = [VP, C.c_int, C.c_int, VP, VP, C.c_int, C.c_double, C.c_int,
                                          C.POINTER(RefResult)]
        L.mtlref_poisson2d_mult.argtypes = [C.c_int, C.c_int, VP, VP, C.c_int]
        L.mtlref_poisson2d_cg.argtypes = [C.c_int, C.c_int, VP, VP, C.c_int, C.c_double, C.POINTER(RefResult)]
        L.mtlref_ell_export.argtypes = [VP, PI, PI, VP, VP]
        L.mtlref_ell_spmv.argtypes = [VP, VP, VP, C.c_int]
        L.mtlref_banded_export.argtypes = [VP, PI, VP, VP]
        L.mtlref_banded_spmv.argtypes = [VP, VP, VP, C.c_int]
        L.mtlref_solve_cyclic.restype = C.c_int
        L.mtlref_solve_cyclic.argtypes = [VP, C.c_int, C.c_int, VP, VP, C.c_int, C.c_double, C.c_int, C.c_int,
                                          C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
        L.mtlref_mm_read.restype = C.c_int
        L.mtlref_mm_read.argtypes = [C.c_char_p, PI, PI, PI, VP, VP, VP]
        _REF[key] = L
    return _REF[key]


def port_lib() -> C.CDLL:
    global _PORT
    if _PORT is None:
        L = C.CDLL(str(PORT_LIB))
        VP = C.c_void_p
        L.mtlo_spmv.argtypes = [C.c_int64, VP, VP, VP, VP, VP, C.c_int]
        L.mtlo_spmv_f32.argtypes = [C.c_int64, VP, VP, VP, VP, VP, C.c_int]
        L.mtlo_dot.restype = C.c_double
        L.mtlo_dot.argtypes = [C.c_int64, VP, VP]
        L.mtlo_ell_spmv.argtypes = [C.c_int64, C.c_int64, C.c_int64, VP, VP, VP, VP, C.c_int]
        L.mtlo_banded_row_kinds.argtypes = [C.c_int64, C.c_int64, C.c_int64, VP, VP]
        L.mtlo_banded_spmv.argtypes = [C.c_int64, C.c_int64, C.c_int64, VP, VP, VP, VP, C.c_int]
        L.mtlo_dot4.restype = C.c_double
        L.mtlo_dot4.argtypes = [C.c_int64, VP, VP]
        L.mtlo_norm4.restype = C.c_double
        L.mtlo_norm4.argtypes = [C.c_int64, VP]
        L.mtlo_pc_apply.argtypes = [C.c_int64, VP, VP, VP, C.c_int, C.c_int, VP, VP]
        L.mtlo_pc_apply_f32.argtypes = [C.c_int64, VP, VP, VP, C.c_int, VP, VP]
        L.mtlo_pc_factor.argtypes = [C.c_int64, VP, VP, VP, C.c_int, C.c_int, C.POINTER(C.c_int64), VP, VP, VP]
        L.mtlo_solve.argtypes = [C.c_int64, VP, VP, VP, C.c_int, C.c_int, VP, VP, C.c_int, C.c_double, C.c_double,
                                 C.c_int, C.c_double, C.POINTER(PortResult)]
        L.mtlo_refine_solve.argtypes = [C.c_int64, VP, VP, VP, C.c_int, C.c_int, VP, VP, C.c_int, C.c_int,
                                        C.c_double, C.c_double, C.POINTER(PortResult)]
        _PORT = L
    return _PORT


class RefMatrix:
    """A CSR held by the reference library (mtl::compressed2D)."""

    def __init__(self, A, omp: bool = False):
        self.L = ref_lib(omp)
        self.A = A
        self.h = self.L.mtlref_csr_create(A.n_rows, A.n_cols, A.nnz, _p(A.row_ptr), _p(A.col), _p(A.val))

    def spmv(self, x, assign=0, y=None):
        x = np.ascontiguousarray(x)
        if x.dtype == np.float32:
            y = np.zeros(self.A.n_rows, np.float32) if y is None else np.array(y, np.float32)
            self.L.mtlref_spmv_f32(self.h, _p(x), _p(y), assign)
        else:
            y = np.zeros(self.A.n_rows) if y is None else np.array(y, np.float64)
            self.L.mtlref_spmv(self.h, _p(x), _p(y), assign)
        return y

    def ell(self):
        """(stride, slots, minor, data) of MTL4's ELL form of A."""
        st, sl = C.c_int64(), C.c_int64()
        self.L.mtlref_ell_export(self.h, C.byref(st), C.byref(sl), None, None)
        mi = np.zeros(st.value * sl.value, np.int64)
        da = np.zeros(st.value * sl.value)
        self.L.mtlref_ell_export(self.h, C.byref(st), C.byref(sl), _p(mi), _p(da))
        return st.value, sl.value, mi, da

    def ell_spmv(self, x, assign=0, y=None):
        y = np.zeros(self.A.n_rows) if y is None else np.array(y, np.float64)
        self.L.mtlref_ell_spmv(self.h, _p(np.ascontiguousarray(x, np.float64)), _p(y), assign)
        return y

    def banded(self):
        """(bands, data) of MTL4's sparse_banded form of A."""
        nb = C.c_int64()
        self.L.mtlref_banded_export(self.h, C.byref(nb), None, None)
        bands = np.zeros(nb.value, np.int64)
        data = np.zeros(self.A.n_rows * nb.value)
        self.L.mtlref_banded_export(self.h, C.byref(nb), _p(bands), _p(data))
        return bands, data

    def banded_spmv(self, x, assign=0, y=None):
        y = np.zeros(self.A.n_rows) if y is None else np.array(y, np.float64)
        self.L.mtlref_banded_spmv(self.h, _p(np.ascontiguousarray(x, np.float64)), _p(y), assign)
        return y

    def spmv_timed(self, x, reps):
        y = np.zeros(self.A.n_rows)
        return self.L.mtlref_spmv_timed(self.h, _p(np.ascontiguousarray(x)), _p(y), reps)

    def pc_apply(self, kind, x, storage_f32=False):
        x = np.ascontiguousarray(x)
        if x.dtype == np.float32:
            y = np.zeros(self.A.n_rows, np.float32)
            self.L.mtlref_pc_apply_f32(self.h, PC_KIND[kind], _p(x), _p(y))
        else:
            y = np.zeros(self.A.n_rows)
            self.L.mtlref_pc_apply(self.h, PC_KIND[kind], int(storage_f32), _p(x), _p(y))
        return y

    def pc_adjoint_apply(self, kind, x, storage_f32=False):
        y = np.zeros(self.A.n_rows)
        if self.L.mtlref_pc_adjoint_apply(self.h, PC_KIND[kind], int(storage_f32),
                                          _p(np.ascontiguousarray(x, np.float64)), _p(y)) != 0:
            raise ValueError(f"no adjoint apply for {kind}")
        return y

    def factors(self, kind):
        nl, nu = C.c_int64(), C.c_int64()
        k = PC_KIND[kind]
        self.L.mtlref_pc_factors(self.h, k, C.byref(nl), None, None, None, C.byref(nu), None, None, None)
        n = self.A.n_rows
        Lrp, Lci, Lv = np.zeros(n + 1, np.int64), np.zeros(nl.value, np.int32), np.zeros(nl.value)
        Urp, Uci, Uv = np.zeros(n + 1, np.int64), np.zeros(nu.value, np.int32), np.zeros(nu.value)
        self.L.mtlref_pc_factors(self.h, k, C.byref(nl), _p(Lrp), _p(Lci), _p(Lv), C.byref(nu), _p(Urp), _p(Uci),
                                 _p(Uv))
        return (Lrp, Lci, Lv), (Urp, Uci, Uv)

    def solve(self, b, solver="cg", pc="identity", max_iter=2000, rtol=1e-8, atol=0.0, restart=0, x0=None,
              pc_f32=False, f32=False):
        r = RefResult()
        if f32:
            b = np.ascontiguousarray(b, np.float32)
            x = np.zeros(self.A.n_rows, np.float32) if x0 is None else np.array(x0, np.float32)
            err = self.L.mtlref_solve_f32(self.h, SOLVER[solver], PC_KIND[pc], _p(b), _p(x), max_iter, rtol, atol,
                                          restart, C.byref(r))
        else:
            b = np.ascontiguousarray(b, np.float64)
            x = np.zeros(self.A.n_rows) if x0 is None else np.array(x0, np.float64)
            err = self.L.mtlref_solve(self.h, SOLVER[solver], PC_KIND[pc], int(pc_f32), _p(b), _p(x), max_iter,
                                      rtol, atol, restart, C.byref(r))
        return {"x": x, "iterations": r.iterations, "error": err, "resid": r.resid, "relresid": r.relresid,
                "setup_s": r.setup_s, "solve_s": r.solve_s}

    def solve_krylov(self, b, solver, pc="identity", max_iter=2000, rtol=1e-8, param=0):
        """FP64 bicg / cgs / tfqmr / qmr / bicgstab_2 / bicgstab_ell / idr_s."""
        r = RefResult()
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.A.n_rows)
        err = self.L.mtlref_solve_krylov(self.h, SOLVER[solver], PC_KIND[pc], _p(b), _p(x), max_iter, rtol, param,
                                         C.byref(r))
        return {"x": x, "iterations": r.iterations, "error": err, "resid": r.resid, "relresid": r.relresid}

    def solve_cyclic(self, b, solver="cg", pc="identity", max_iter=2000, rtol=1e-8, cycle=100, multi_print=False):
        """FP64 solve with itl::cyclic_iteration printing into a string;
        returns (error, text)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.A.n_rows)
        need = C.c_size_t()
        args = [self.h, SOLVER[solver], PC_KIND[pc], _p(b), None, max_iter, rtol, cycle, int(multi_print)]
        self.L.mtlref_solve_cyclic(*args[:4], _p(x), *args[5:], None, 0, C.byref(need))
        buf = C.create_string_buffer(need.value)
        x[:] = 0
        err = self.L.mtlref_solve_cyclic(*args[:4], _p(x), *args[5:], buf, need.value, None)
        return err, buf.value.decode()

    def refine(self, b, solver="cg", pc="ic_0", max_outer=20, max_inner=2000, rtol=1e-8, inner_rtol=1e-4):
        r = RefResult()
        x = np.zeros(self.A.n_rows)
        err = self.L.mtlref_refine_solve(self.h, SOLVER[solver], PC_KIND[pc], _p(np.ascontiguousarray(b)), _p(x),
                                         max_outer, max_inner, rtol, inner_rtol, 0, C.byref(r))
        return {"x": x, "iterations": r.iterations, "outer": r.outer, "error": err, "resid": r.resid,
                "relresid": r.relresid, "setup_s": r.setup_s, "solve_s": r.solve_s}

    def __del__(self):
        try:
            self.L.mtlref_csr_destroy(self.h)
        except Exception:
            pass


def ref_laplacian(m, n):
    L = ref_lib()
    nnz = C.c_int64()
    L.mtlref_laplacian_setup(m, n, C.byref(nnz), None, None, None)
    rp, ci, v = np.zeros(m * n + 1, np.int64), np.zeros(nnz.value, np.int32), np.zeros(nnz.value)
    L.mtlref_laplacian_setup(m, n, C.byref(nnz), _p(rp), _p(ci), _p(v))
    return rp, ci, v


# ----------------------------------------------------------------- restatement
def port_spmv(A, x, assign=0, y=None, val=None):
    L = port_lib()
    x = np.ascontiguousarray(x)
    if x.dtype == np.float32:
        v = np.ascontiguousarray(A.val if val is None else val, np.float32)
        y = np.zeros(A.n_rows, np.float32) if y is None else np.array(y, np.float32)
        L.mtlo_spmv_f32(A.n_rows, _p(A.row_ptr), _p(A.col), _p(v), _p(x), _p(y), assign)
    else:
        y = np.zeros(A.n_rows) if y is None else np.array(y, np.float64)
        L.mtlo_spmv(A.n_rows, _p(A.row_ptr), _p(A.col), _p(A.val), _p(x), _p(y), assign)
    return y


def port_pc_apply(A, kind, x, storage_f32=False):
    L = port_lib()
    x = np.ascontiguousarray(x)
    if x.dtype == np.float32:
        y = np.zeros(A.n_rows, np.float32)
        L.mtlo_pc_apply_f32(A.n_rows, _p(A.row_ptr), _p(A.col), _p(A.val), PC_KIND[kind], _p(x), _p(y))
    else:
        y = np.zeros(A.n_rows)
        L.mtlo_pc_apply(A.n_rows, _p(A.row_ptr), _p(A.col), _p(A.val), PC_KIND[kind], int(storage_f32), _p(x),
                        _p(y))
    return y


def port_factor(A, kind, which):
    L = port_lib()
    nnz = C.c_int64()
    w = 0 if which == "L" else 1
    L.mtlo_pc_factor(A.n_rows, _p(A.row_ptr), _p(A.col), _p(A.val), PC_KIND[kind], w, C.byref(nnz), None, None, None)
    rp, ci, v = np.zeros(A.n_rows + 1, np.int64), np.zeros(nnz.value, np.int32), np.zeros(nnz.value)
    L.mtlo_pc_factor(A.n_rows, _p(A.row_ptr), _p(A.col), _p(A.val), PC_KIND[kind], w, C.byref(nnz), _p(rp), _p(ci),
                     _p(v))
    return rp, ci, v


def port_solve(A, b, solver="cg", pc="identity", max_iter=2000, rtol=1e-8, atol=0.0, restart=0, norm_r0=-1.0):
    L = port_lib()
    r = PortResult()
    x = np.zeros(A.n_rows)
    b = np.ascontiguousarray(b, np.float64)
    err = L.mtlo_solve(A.n_rows, _p(A.row_ptr), _p(A.col), _p(A.val), SOLVER[solver], PC_KIND[pc], _p(b), _p(x),
                       max_iter, rtol, atol, restart, norm_r0, C.byref(r))
    return {"x": x, "iterations": r.iterations, "error": err, "resid": r.resid, "relresid": r.relresid}


def port_refine(A, b, solver="cg", pc="ic_0", max_outer=20, max_inner=2000, rtol=1e-8, inner_rtol=1e-4):
    L = port_lib()
    r = PortResult()
    x = np.zeros(A.n_rows)
    err = L.mtlo_refine_solve(A.n_rows, _p(A.row_ptr), _p(A.col), _p(A.val), SOLVER[solver], PC_KIND[pc],
                              _p(np.ascontiguousarray(b)), _p(x), max_outer, max_inner, rtol, inner_rtol,
                              C.byref(r))
    return {"x": x, "iterations": r.iterations, "outer": r.outer, "error": err, "resid": r.resid,
            "relresid": r.relresid}


def solve(A, b, solver="cg", pc="identity", **kw):
    """Reference solve when the reference-built library is present, else the
    restatement."""
    if ref_available():
        return RefMatrix(A).solve(b, solver, pc, **kw)
    return port_solve(A, b, solver, pc, **kw)


def ref_matrix_market(path):
    """(status, (n_rows, n_cols, row_ptr, col, val)) as the reference's
    matrix_market_istream reads the file; status 1: file_not_found, 2: other
    exception."""
    L = ref_lib()
    nr, nc, nz = C.c_int64(), C.c_int64(), C.c_int64()
    p = str(path).encode()
    st = L.mtlref_mm_read(p, C.byref(nr), C.byref(nc), C.byref(nz), None, None, None)
    if st:
        return st, None
    rp = np.zeros(nr.value + 1, np.int64)
    ci = np.zeros(nz.value, np.int32)
    v = np.zeros(nz.value)
    L.mtlref_mm_read(p, C.byref(nr), C.byref(nc), C.byref(nz), _p(rp), _p(ci), _p(v))
    return 0, (nr.value, nc.value, rp, ci, v)


def port_ell_spmv(n_rows, stride, slots, minor, data, x, assign=0, y=None):
    L = port_lib()
    y = np.zeros(n_rows) if y is None else np.array(y, np.float64)
    mi = np.ascontiguousarray(minor, np.int64)
    da = np.ascontiguousarray(data, np.float64)
    L.mtlo_ell_spmv(n_rows, stride, slots, _p(mi), _p(da), _p(np.ascontiguousarray(x, np.float64)), _p(y), assign)
    return y


def port_banded_spmv(n_rows, n_cols, bands, data, x, assign=0, y=None):
    L = port_lib()
    y = np.zeros(n_rows) if y is None else np.array(y, np.float64)
    b = np.ascontiguousarray(bands, np.int64)
    da = np.ascontiguousarray(data, np.float64)
    L.mtlo_banded_spmv(n_rows, n_cols, b.size, _p(b), _p(da), _p(np.ascontiguousarray(x, np.float64)), _p(y), assign)
    return y


def ref_poisson2d_mult(m, n, x, assign=0, y=None):
    y = np.zeros(m * n) if y is None else np.array(y, np.float64)
    ref_lib().mtlref_poisson2d_mult(m, n, _p(np.ascontiguousarray(x, np.float64)), _p(y), assign)
    return y


def ref_poisson2d_cg(m, n, b, max_iter=2000, rtol=1e-8):
    r = RefResult()
    x = np.zeros(m * n)
    err = ref_lib().mtlref_poisson2d_cg(m, n, _p(np.ascontiguousarray(b, np.float64)), _p(x), max_iter, rtol,
                                        C.byref(r))
    return {"x": x, "iterations": r.iterations, "error": err, "relresid": r.relresid}
