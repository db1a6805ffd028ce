"""ctypes binding of libmtl4_b200.so (the C ABI in include/mtl4_b200/mtlg.h).

The shared library is built in-tree by ``mtl4_b200.build``.  There is no CPU
fallback: if the library is missing or fails to load, importing the package's
solver API raises ``ImportError``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmtl4_b200.so"

# status codes (mtlg.h)
OK = 0
ERR_INVALID_ARG = 1
ERR_NOT_SQUARE = 2
ERR_MISSING_DIAGONAL = 3
ERR_ZERO_PIVOT = 4
ERR_BREAKDOWN = 5
ERR_OOM = 6
ERR_TIMEOUT = 7
ERR_CUDA = 8
ERR_INCOMPATIBLE_SIZE = 9
ERR_UNSORTED = 10
ERR_TOO_LARGE = 11
ERR_NOT_SUPPORTED = 12
ERR_ADMISSION = 13
ERR_NOT_FOUND = 14
PENDING = 15
ERR_FILE_NOT_FOUND = 16
ERR_FORMAT = 17

F64, F32 = 0, 1
ASSIGN, PLUS, MINUS = 0, 1, 2
PC_IDENTITY, PC_DIAGONAL, PC_ILU0, PC_IC0 = 0, 1, 2, 3
CG, BICGSTAB, GMRES = 0, 1, 2
BICG, CGS, TFQMR, QMR, BICGSTAB_2, BICGSTAB_ELL, IDR_S = 3, 4, 5, 6, 7, 8, 9
ST_RUNNING, ST_CONVERGED, ST_MAXIT, ST_BREAKDOWN, ST_NO_DIRECTION, ST_STALLED = 0, 1, 2, 3, 4, 5


class IterParams(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("restart", C.c_int), ("rtol", C.c_double), ("atol", C.c_double),
                ("norm_r0", C.c_double)]


class IterResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("error_code", C.c_int), ("status", C.c_int),
                ("outer_iterations", C.c_int), ("resid", C.c_double), ("relresid", C.c_double),
                ("norm_r0", C.c_double), ("seconds", C.c_double), ("fp64_fallback", C.c_int),
                ("reserved", C.c_int)]


class RefineParams(C.Structure):
    _fields_ = [("max_outer", C.c_int), ("max_inner", C.c_int), ("restart", C.c_int), ("pad", C.c_int),
                ("rtol", C.c_double), ("inner_rtol", C.c_double)]


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget", C.c_size_t), ("max_active", C.c_int), ("iters_per_step", C.c_int),
                ("precision", C.c_int), ("pad", C.c_int), ("rtol", C.c_double), ("inner_rtol", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64),
                ("rejected", C.c_int64), ("cancelled", C.c_int64), ("active", C.c_int64),
                ("queued", C.c_int64), ("steps", C.c_int64), ("bytes_in_use", C.c_size_t)]


VP = C.c_void_p
I64 = C.c_int64
PI64 = C.POINTER(C.c_int64)
PINT = C.POINTER(C.c_int)
PDBL = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "mtlg_ctx_create": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(VP)]),
    "mtlg_ctx_destroy": (C.c_int, [VP]),
    "mtlg_ctx_synchronize": (C.c_int, [VP]),
    "mtlg_ctx_set_stream": (C.c_int, [VP, VP]),
    "mtlg_ctx_stream": (VP, [VP]),
    "mtlg_ctx_kernel_launches": (I64, [VP]),
    "mtlg_ctx_bytes_in_use": (C.c_size_t, [VP]),
    "mtlg_ctx_set_tuning": (C.c_int, [VP, C.c_char_p, I64]),
    "mtlg_ctx_get_tuning": (C.c_int, [VP, C.c_char_p, PI64]),
    "mtlg_status_string": (C.c_char_p, [C.c_int]),
    "mtlg_last_error_message": (C.c_char_p, []),
    "mtlg_csr_create": (C.c_int, [VP, I64, I64, I64, VP, VP, VP, C.c_int, C.POINTER(VP)]),
    "mtlg_csr_destroy": (C.c_int, [VP]),
    "mtlg_csr_info": (C.c_int, [VP, PI64, PI64, PI64]),
    "mtlg_csr_update_values": (C.c_int, [VP, VP, C.c_int]),
    "mtlg_csr_plan_info": (C.c_int, [VP, PI64, PINT]),
    "mtlg_vec_create": (C.c_int, [VP, I64, C.c_int, C.POINTER(VP)]),
    "mtlg_vec_wrap": (C.c_int, [VP, I64, C.c_int, VP, C.POINTER(VP)]),
    "mtlg_vec_destroy": (C.c_int, [VP]),
    "mtlg_vec_upload": (C.c_int, [VP, VP, I64]),
    "mtlg_vec_download": (C.c_int, [VP, VP, I64]),
    "mtlg_vec_fill": (C.c_int, [VP, C.c_double]),
    "mtlg_vec_device_ptr": (VP, [VP]),
    "mtlg_vec_size": (I64, [VP]),
    "mtlg_spmv": (C.c_int, [VP, VP, VP, VP, C.c_int]),
    "mtlg_spmv_dot": (C.c_int, [VP, VP, VP, VP, PDBL]),
    "mtlg_spmv_dot_noalloc": (C.c_int, [I64, I64, VP, VP, VP, VP, VP, VP, VP]),
    "mtlg_spmv_gather_floor": (C.c_int, [VP, VP, VP]),
    "mtlg_dot": (C.c_int, [VP, VP, VP, PDBL]),
    "mtlg_two_norm": (C.c_int, [VP, VP, PDBL]),
    "mtlg_axpy": (C.c_int, [VP, C.c_double, VP, VP]),
    "mtlg_pc_create": (C.c_int, [VP, VP, C.c_int, C.c_int, C.POINTER(VP)]),
    "mtlg_pc_destroy": (C.c_int, [VP]),
    "mtlg_pc_apply": (C.c_int, [VP, VP, VP, VP]),
    "mtlg_pc_adjoint_apply": (C.c_int, [VP, VP, VP, VP]),
    "mtlg_pc_factor": (C.c_int, [VP, C.c_int, PI64, VP, VP, VP]),
    "mtlg_pc_levels": (C.c_int, [VP, PINT, PINT]),
    "mtlg_pc_sweep_plan": (C.c_int, [VP, VP, C.c_int, PINT]),
    "mtlg_grid_structure": (C.c_int, [I64, VP, VP, C.c_int, PINT]),
    "mtlg_solve": (C.c_int, [VP, C.c_int, VP, VP, VP, VP, VP, C.POINTER(IterParams), C.POINTER(IterResult)]),
    "mtlg_refine_solve": (C.c_int, [VP, C.c_int, VP, VP, VP, VP, C.POINTER(RefineParams), C.POINTER(IterResult)]),
    "mtlg_batch_create": (C.c_int, [VP, C.POINTER(VP)]),
    "mtlg_batch_destroy": (C.c_int, [VP]),
    "mtlg_batch_add": (C.c_int, [VP, I64, I64, VP, VP, VP, VP, C.c_int, C.c_int, C.POINTER(IterParams), PINT]),
    "mtlg_batch_solve": (C.c_int, [VP, C.c_int, C.POINTER(RefineParams)]),
    "mtlg_batch_result": (C.c_int, [VP, C.c_int, VP, C.POINTER(IterResult)]),
    "mtlg_batch_size": (C.c_int, [VP]),
    "mtlg_partition_systems": (C.c_int, [C.c_int64, VP, C.c_int, VP, VP]),
    "mtlg_trace_enable": (C.c_int, [C.c_int]),
    "mtlg_poisson2d_spmv": (C.c_int, [VP, C.c_int, C.c_int, VP, VP, C.c_int]),
    "mtlg_poisson2d_solve": (C.c_int, [VP, C.c_int, C.c_int, C.c_int, VP, VP, VP, VP]),
    "mtlg_ell_create": (C.c_int, [VP, C.c_int64, C.c_int64, C.c_int64, C.c_int64, VP, VP, C.c_int, C.POINTER(VP)]),
    "mtlg_ell_destroy": (C.c_int, [VP]),
    "mtlg_ell_spmv": (C.c_int, [VP, VP, VP, VP, C.c_int]),
    "mtlg_banded_create": (C.c_int, [VP, C.c_int64, C.c_int64, C.c_int64, VP, VP, C.c_int, C.POINTER(VP)]),
    "mtlg_banded_destroy": (C.c_int, [VP]),
    "mtlg_banded_spmv": (C.c_int, [VP, VP, VP, VP, C.c_int]),
    "mtlg_ctx_set_residual_log": (C.c_int, [VP, C.c_int]),
    "mtlg_ctx_residual_log": (C.c_int, [VP, VP, C.c_int, C.POINTER(C.c_int)]),
    "mtlg_server_admission": (C.c_int, [C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t]),
    "mtlg_mm_read": (C.c_int, [VP, C.c_char_p, C.POINTER(VP)]),
    "mtlg_mm_read_host": (C.c_int, [C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                    VP, VP, VP]),
    "mtlg_trace_reset": (C.c_int, []),
    "mtlg_trace_report": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "mtlg_server_create": (C.c_int, [VP, C.POINTER(ServerOpts), C.POINTER(VP)]),
    "mtlg_server_destroy": (C.c_int, [VP]),
    "mtlg_server_submit": (C.c_int, [VP, I64, I64, VP, VP, VP, VP, C.c_int, C.c_int, C.c_int, PI64]),
    "mtlg_server_step": (C.c_int, [VP]),
    "mtlg_server_poll": (C.c_int, [VP, I64, VP, C.POINTER(IterResult)]),
    "mtlg_server_cancel": (C.c_int, [VP, I64]),
    "mtlg_server_stats_get": (C.c_int, [VP, C.POINTER(ServerStats)]),
}


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB


class MtlError(RuntimeError):
    """Base of the errors the C ABI reports (mtl::runtime_error)."""
    status = -1


class logic_error(MtlError):
    pass


class matrix_not_square(MtlError):
    status = ERR_NOT_SQUARE


class missing_diagonal(MtlError):
    status = ERR_MISSING_DIAGONAL


class incompatible_size(MtlError):
    status = ERR_INCOMPATIBLE_SIZE


class unexpected_orthogonality(MtlError):
    """itl::unexpected_orthogonality (BiCGSTAB breakdown)."""
    status = ERR_BREAKDOWN


class device_timeout(MtlError):
    status = ERR_TIMEOUT


class out_of_memory(MtlError):
    status = ERR_OOM


class file_not_found(MtlError):
    """mtl::io::file_not_found (io/matrix_market.hpp:53-58)."""
    status = ERR_FILE_NOT_FOUND


class runtime_error(MtlError):
    """mtl::runtime_error, e.g. a malformed Matrix Market file."""
    status = ERR_FORMAT


_EXC = {
    ERR_NOT_SQUARE: matrix_not_square,
    ERR_MISSING_DIAGONAL: missing_diagonal,
    ERR_INCOMPATIBLE_SIZE: incompatible_size,
    ERR_BREAKDOWN: unexpected_orthogonality,
    ERR_TIMEOUT: device_timeout,
    ERR_OOM: out_of_memory,
    ERR_INVALID_ARG: logic_error,
    ERR_UNSORTED: logic_error,
    ERR_FILE_NOT_FOUND: file_not_found,
    ERR_FORMAT: runtime_error,
}


def check(status: int, what: str = "") -> int:
    if status in (OK, PENDING):
        return status
    L = lib()
    msg = L.mtlg_status_string(status).decode()
    detail = (L.mtlg_last_error_message() or b"").decode()
    exc = _EXC.get(status, MtlError)
    e = exc(f"{what}: {msg}" + (f" ({detail})" if detail else ""))
    e.status = status
    raise e
