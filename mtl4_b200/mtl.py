"""Python mirror of MTL4's storage types and vector operations on the GPU.

``compressed2D`` and ``dense_vector`` keep their data in device memory owned by
the C ABI (include/mtl4_b200/mtlg.h).  Names and argument meanings follow
boost/numeric/mtl (compressed2D.hpp:259,355; dense_vector.hpp:52,122;
operation/dot.hpp:228; operation/two_norm.hpp:54;
vector/crtp_base_vector.hpp:94-101 for w = A*v, w += A*v, w -= A*v).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check

_DT = {np.dtype(np.float64): _lib.F64, np.dtype(np.float32): _lib.F32}


class context:
    """One device, one stream.  Not thread-safe (as the reference's ILU/IC
    apply is not re-entrant, itl/pc/ilu.hpp:76)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self._L = _lib.lib()
        h = C.c_void_p()
        check(self._L.mtlg_ctx_create(device, hbm_budget, C.byref(h)), "ctx_create")
        self.h = h
        self.device = device
        self.autotune = None   # autotune.Cache when launch shapes are tuned per operator class

    def enable_autotune(self, cache=None):
        """Tunes launch shapes per operator class from now on: preconditioner
        set-ups take the chunked-sweep settings of their operator, solves the
        vector-pass setting and mult the SpMV kernel (measured once per class,
        then read from `cache`, an autotune.Cache or a path)."""
        from . import autotune
        if cache is None or isinstance(cache, (str, bytes)) or hasattr(cache, "__fspath__"):
            cache = autotune.Cache(cache) if cache is not None else autotune.Cache()
        self.autotune = cache

    def disable_autotune(self):
        self.autotune = None

    def synchronize(self):
        check(self._L.mtlg_ctx_synchronize(self.h), "synchronize")

    def kernel_launches(self) -> int:
        return int(self._L.mtlg_ctx_kernel_launches(self.h))

    def bytes_in_use(self) -> int:
        return int(self._L.mtlg_ctx_bytes_in_use(self.h))

    def set_tuning(self, key: str, value: int):
        check(self._L.mtlg_ctx_set_tuning(self.h, key.encode(), int(value)), "set_tuning")

    def get_tuning(self, key: str) -> int:
        v = C.c_int64()
        check(self._L.mtlg_ctx_get_tuning(self.h, key.encode(), C.byref(v)), "get_tuning")
        return v.value

    def ensure_residual_log(self, tests: int):
        """Device residual log of at least `tests` termination tests."""
        if tests > getattr(self, "_log_cap", 0):
            check(self._L.mtlg_ctx_set_residual_log(self.h, int(tests)), "residual log")
            self._log_cap = int(tests)

    def residual_log(self):
        """(iteration, residual) pairs of the last CG / BiCGSTAB solve as a flat
        array, or None when the log overflowed."""
        n = C.c_int()
        check(self._L.mtlg_ctx_residual_log(self.h, None, 0, C.byref(n)), "residual log")
        if n.value > getattr(self, "_log_cap", 0):
            return None
        out = np.zeros(2 * n.value)
        if n.value:
            check(self._L.mtlg_ctx_residual_log(self.h, _ptr(out), n.value, C.byref(n)), "residual log")
        return out

    def set_stream(self, cuda_stream_ptr: int | None):
        check(self._L.mtlg_ctx_set_stream(self.h, C.c_void_p(cuda_stream_ptr or 0)), "set_stream")

    def close(self):
        if getattr(self, "h", None):
            self._L.mtlg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_DEFAULT: dict[int, context] = {}


def default_context(device: int = 0) -> context:
    if device not in _DEFAULT:
        _DEFAULT[device] = context(device)
    return _DEFAULT[device]


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class compressed2D:
    """CSR matrix on the device (row_ptr int64 on the host side, int32 on the
    device; sorted, distinct, in-range columns in every row)."""

    def __init__(self, row_ptr, col, val, shape=None, ctx: context | None = None):
        self.ctx = ctx or default_context()
        rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
        ci = np.ascontiguousarray(col, dtype=np.int32)
        v = np.asarray(val)
        if v.dtype not in _DT:
            v = v.astype(np.float64)
        v = np.ascontiguousarray(v)
        n_rows = rp.size - 1
        n_cols = shape[1] if shape is not None else n_rows
        h = C.c_void_p()
        check(self.ctx._L.mtlg_csr_create(self.ctx.h, n_rows, n_cols, int(rp[-1]), _ptr(rp), _ptr(ci), _ptr(v),
                                          _DT[v.dtype], C.byref(h)), "compressed2D")
        self.h = h
        self.shape = (n_rows, n_cols)
        self.nnz = int(rp[-1])
        self.host_row_ptr = rp   # for the autotuner's operator key
        self._tuned = {}

    @classmethod
    def from_problem(cls, A, ctx: context | None = None) -> "compressed2D":
        return cls(A.row_ptr, A.col, A.val, (A.n_rows, A.n_cols), ctx)

    @classmethod
    def from_matrix_market(cls, path, ctx: context | None = None) -> "compressed2D":
        """A = mtl::io::matrix_market(path) straight into device CSR (FP64)."""
        self = cls.__new__(cls)
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        check(self.ctx._L.mtlg_mm_read(self.ctx.h, str(path).encode(), C.byref(h)), "matrix_market")
        self.h = h
        nr, nc, nz = C.c_int64(), C.c_int64(), C.c_int64()
        check(self.ctx._L.mtlg_csr_info(h, C.byref(nr), C.byref(nc), C.byref(nz)), "csr_info")
        self.shape = (nr.value, nc.value)
        self.nnz = nz.value
        self.host_row_ptr = None
        self._tuned = {}
        return self

    def num_rows(self) -> int:
        return self.shape[0]

    def num_cols(self) -> int:
        return self.shape[1]

    def plan_info(self):
        k = (C.c_int64 * 3)()
        mr = C.c_int()
        check(self.ctx._L.mtlg_csr_plan_info(self.h, k, C.byref(mr)), "plan_info")
        return {"stream_tiles": k[0], "long_tiles": k[1], "max_row": mr.value}

    def update_values(self, val):
        v = np.ascontiguousarray(val)
        check(self.ctx._L.mtlg_csr_update_values(self.h, _ptr(v), _DT[v.dtype]), "update_values")

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                self.ctx._L.mtlg_csr_destroy(self.h)
        except Exception:
            pass

    def __mul__(self, v: "dense_vector") -> "_MatVec":
        return _MatVec(self, v)


class _MatVec:
    """Lazy A*v, consumed by dense_vector.assign / += / -= as the reference's
    mat_cvec_times_expr is."""

    def __init__(self, A, v):
        self.A, self.v = A, v


class dense_vector:
    """Device vector of float64 or float32."""

    def __init__(self, n_or_array, dtype=np.float64, ctx: context | None = None, _wrap_ptr: int | None = None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        if isinstance(n_or_array, (int, np.integer)):
            n = int(n_or_array)
            self.dtype = np.dtype(dtype)
            if _wrap_ptr is not None:
                check(self.ctx._L.mtlg_vec_wrap(self.ctx.h, n, _DT[self.dtype], C.c_void_p(_wrap_ptr), C.byref(h)),
                      "dense_vector")
            else:
                check(self.ctx._L.mtlg_vec_create(self.ctx.h, n, _DT[self.dtype], C.byref(h)), "dense_vector")
            self.h = h
            self.n = n
        else:
            a = np.asarray(n_or_array)
            self.dtype = np.dtype(dtype) if dtype is not None else a.dtype
            a = np.ascontiguousarray(a, dtype=self.dtype)
            self.n = a.size
            check(self.ctx._L.mtlg_vec_create(self.ctx.h, self.n, _DT[self.dtype], C.byref(h)), "dense_vector")
            self.h = h
            self.upload(a)

    def __len__(self):
        return self.n

    def size(self) -> int:
        return self.n

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        check(self.ctx._L.mtlg_vec_upload(self.h, _ptr(a), a.size), "upload")

    def numpy(self) -> np.ndarray:
        out = np.empty(self.n, dtype=self.dtype)
        check(self.ctx._L.mtlg_vec_download(self.h, _ptr(out), self.n), "download")
        return out

    def fill(self, value: float):
        check(self.ctx._L.mtlg_vec_fill(self.h, float(value)), "fill")

    def device_ptr(self) -> int:
        return int(self.ctx._L.mtlg_vec_device_ptr(self.h) or 0)

    def assign(self, e: _MatVec):
        mult(e.A, e.v, self, "=")
        return self

    def __iadd__(self, e):
        if isinstance(e, _MatVec):
            mult(e.A, e.v, self, "+=")
            return self
        return NotImplemented

    def __isub__(self, e):
        if isinstance(e, _MatVec):
            mult(e.A, e.v, self, "-=")
            return self
        return NotImplemented

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                self.ctx._L.mtlg_vec_destroy(self.h)
        except Exception:
            pass


_ASSIGN = {"=": _lib.ASSIGN, "+=": _lib.PLUS, "-=": _lib.MINUS}


def ell_layout(A):
    """MTL4's ELL form of a host CSR (matrix/ell_matrix.hpp:127-170): stride =
    rows rounded up to 32, slots = the longest row, entry j of row r at
    r + j * stride; short rows padded with value 0 at their last column (0
    for an empty row).  Returns (stride, slots, minor, data)."""
    n = A.n_rows
    lens = np.diff(A.row_ptr)
    slots = int(lens.max()) if n else 0
    stride = (n + 31) // 32 * 32
    minor = np.zeros(slots * stride, np.int64)
    data = np.zeros(slots * stride)
    for j in range(slots):
        has = lens > j
        k = j * stride + np.arange(n)
        e = A.row_ptr[:-1] + np.minimum(j, np.maximum(lens - 1, 0))
        last = np.where(lens > 0, A.col[np.minimum(e, max(A.nnz - 1, 0))] if A.nnz else 0, 0)
        minor[k] = last
        data[k] = np.where(has, A.val[np.minimum(A.row_ptr[:-1] + j, max(A.nnz - 1, 0))] if A.nnz else 0.0, 0.0)
    return stride, slots, minor, data


def banded_layout(A):
    """MTL4's sparse_banded form of a host CSR: the distinct offsets col - row
    in increasing order and one value per band and row, row by row (0 where a
    row has no entry on a band).  Returns (bands, data)."""
    rows = np.repeat(np.arange(A.n_rows), np.diff(A.row_ptr))
    off = A.col.astype(np.int64) - rows
    bands = np.unique(off)
    data = np.zeros(A.n_rows * bands.size)
    data[rows * bands.size + np.searchsorted(bands, off)] = A.val
    return bands, data


class ell_matrix:
    """mtl::mat::ell_matrix on the device (its own layout; see ell_layout)."""

    def __init__(self, n_rows, n_cols, slots, stride, minor, data, ctx: context | None = None):
        self.ctx = ctx or default_context()
        mi = np.ascontiguousarray(minor, np.int64)
        v = np.ascontiguousarray(data)
        if v.dtype not in _DT:
            v = v.astype(np.float64)
        h = C.c_void_p()
        check(self.ctx._L.mtlg_ell_create(self.ctx.h, int(n_rows), int(n_cols), int(slots), int(stride), _ptr(mi),
                                          _ptr(v), _DT[v.dtype], C.byref(h)), "ell_matrix")
        self.h = h
        self.shape = (int(n_rows), int(n_cols))

    @classmethod
    def from_csr(cls, A, ctx: context | None = None) -> "ell_matrix":
        st, sl, mi, da = ell_layout(A)
        return cls(A.n_rows, A.n_cols, sl, st, mi, da, ctx)

    def __mul__(self, v: "dense_vector") -> "_MatVec":
        return _MatVec(self, v)

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                self.ctx._L.mtlg_ell_destroy(self.h)
        except Exception:
            pass


class sparse_banded:
    """mtl::mat::sparse_banded on the device (values kept band by band)."""

    def __init__(self, n_rows, n_cols, bands, data, ctx: context | None = None):
        self.ctx = ctx or default_context()
        b = np.ascontiguousarray(bands, np.int64)
        v = np.ascontiguousarray(data)
        if v.dtype not in _DT:
            v = v.astype(np.float64)
        h = C.c_void_p()
        check(self.ctx._L.mtlg_banded_create(self.ctx.h, int(n_rows), int(n_cols), b.size, _ptr(b), _ptr(v),
                                             _DT[v.dtype], C.byref(h)), "sparse_banded")
        self.h = h
        self.shape = (int(n_rows), int(n_cols))

    @classmethod
    def from_csr(cls, A, ctx: context | None = None) -> "sparse_banded":
        bands, data = banded_layout(A)
        return cls(A.n_rows, A.n_cols, bands, data, ctx)

    def __mul__(self, v: "dense_vector") -> "_MatVec":
        return _MatVec(self, v)

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                self.ctx._L.mtlg_banded_destroy(self.h)
        except Exception:
            pass


class poisson2D_dirichlet:
    """Matrix-free 2D Poisson operator on an m x n grid (the reference's
    mtl::mat::poisson2D_dirichlet, matrix/poisson2D_dirichlet.hpp:24-80)."""

    def __init__(self, m: int, n: int, ctx: context | None = None):
        self.ctx = ctx or default_context()
        self.m, self.n = int(m), int(n)
        self.shape = (self.m * self.n, self.m * self.n)

    def num_rows(self) -> int:
        return self.m * self.n

    def __mul__(self, v: "dense_vector") -> "_MatVec":
        return _MatVec(self, v)


def tuned(A, what: str, tune):
    """Applies the autotuned settings `what` of device matrix A (measured on
    first use per operator class; kept on A) when its context tunes."""
    ctx = A.ctx
    if ctx.autotune is None or not isinstance(A, compressed2D):
        return
    from . import autotune
    key = what if isinstance(what, str) else tuple(what)
    choice = A._tuned.get(key)
    if choice is None:
        choice = tune(ctx, A, ctx.autotune)[0]
        A._tuned[key] = choice
    autotune.apply_settings(ctx, choice)


def mult(A, x: dense_vector, y: dense_vector, assign: str = "=", tune: bool = True):
    """y = A x, y += A x or y -= A x (A: compressed2D, ell_matrix or
    sparse_banded)."""
    if tune and isinstance(A, compressed2D) and A.ctx.autotune is not None:
        from . import autotune
        tuned(A, "spmv", lambda ctx, Ad, cache: autotune.tune_spmv(ctx, Ad, cache))
    if isinstance(A, poisson2D_dirichlet):
        check(A.ctx._L.mtlg_poisson2d_spmv(A.ctx.h, A.m, A.n, x.h, y.h, _ASSIGN[assign]), "mult")
    elif isinstance(A, ell_matrix):
        check(A.ctx._L.mtlg_ell_spmv(A.ctx.h, A.h, x.h, y.h, _ASSIGN[assign]), "mult")
    elif isinstance(A, sparse_banded):
        check(A.ctx._L.mtlg_banded_spmv(A.ctx.h, A.h, x.h, y.h, _ASSIGN[assign]), "mult")
    else:
        check(A.ctx._L.mtlg_spmv(A.ctx.h, A.h, x.h, y.h, _ASSIGN[assign]), "mult")


def gather_floor(A: compressed2D, x: dense_vector):
    """Roofline probe: stream A's values and columns and gather x[col] for
    every entry, without the row structure (the memory floor of mult on A);
    asynchronous, to be timed by the caller."""
    check(A.ctx._L.mtlg_spmv_gather_floor(A.ctx.h, A.h, x.h), "gather_floor")


def mult_dot(A: compressed2D, p: dense_vector, q: dense_vector) -> float:
    """(q = A p) || (alpha = dot(p, q)) in one pass (cg.hpp:103)."""
    out = C.c_double()
    check(A.ctx._L.mtlg_spmv_dot(A.ctx.h, A.h, p.h, q.h, C.byref(out)), "mult_dot")
    return out.value


def dot(x: dense_vector, y: dense_vector) -> float:
    out = C.c_double()
    check(x.ctx._L.mtlg_dot(x.ctx.h, x.h, y.h, C.byref(out)), "dot")
    return out.value


def two_norm(x: dense_vector) -> float:
    out = C.c_double()
    check(x.ctx._L.mtlg_two_norm(x.ctx.h, x.h, C.byref(out)), "two_norm")
    return out.value


def axpy(a: float, x: dense_vector, y: dense_vector):
    check(x.ctx._L.mtlg_axpy(x.ctx.h, float(a), x.h, y.h), "axpy")


def read_matrix_market(path):
    """Host CSR of a Matrix Market file as the library's reader parses it
    (mtl4_b200.problems.CSR; needs no GPU)."""
    from .problems import CSR
    L = _lib.lib()
    nr, nc, nz = C.c_int64(), C.c_int64(), C.c_int64()
    p = str(path).encode()
    check(L.mtlg_mm_read_host(p, C.byref(nr), C.byref(nc), C.byref(nz), None, None, None), "matrix_market")
    rp = np.zeros(nr.value + 1, np.int64)
    ci = np.zeros(nz.value, np.int32)
    v = np.zeros(nz.value, np.float64)
    check(L.mtlg_mm_read_host(p, C.byref(nr), C.byref(nc), C.byref(nz), _ptr(rp), _ptr(ci), _ptr(v)),
          "matrix_market")
    return CSR(nr.value, nc.value, rp, ci, v)
