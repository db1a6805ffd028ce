"""The C-ABI library loads and exports every symbol include/mtl4_b200/mtlg.h
declares (no compute calls: runs without a GPU)."""
import ctypes
import re

from conftest import ROOT


def declared_symbols():
    text = (ROOT / "include" / "mtl4_b200" / "mtlg.h").read_text()
    return sorted(set(re.findall(r"\b(mtlg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "mtlg_solve" in syms and "mtlg_spmv" in syms and len(syms) > 40


def test_library_exports_every_declared_symbol():
    from mtl4_b200 import _lib
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_signatures_cover_header():
    from mtl4_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_status_strings_need_no_gpu():
    from mtl4_b200 import _lib
    L = _lib.load()
    assert L.mtlg_status_string(0) == b"ok"
    assert b"orthogonality" in L.mtlg_status_string(_lib.ERR_BREAKDOWN)


def test_missing_library_fails_loudly(tmp_path):
    import pytest
    from mtl4_b200 import _lib
    with pytest.raises(ImportError):
        _lib.load(tmp_path / "nope.so")


def test_noalloc_rejects_null_matrix_arrays_without_touching_the_gpu():
    # argument checks run before any CUDA call, so this needs no GPU
    import ctypes as C
    from mtl4_b200 import _lib
    L = _lib.load()
    buf = (C.c_double * 8)()
    ok = C.cast(buf, C.c_void_p)
    for missing in range(5):
        args = [ok] * 5
        args[missing] = None   # row_ptr, col, val, p, q in turn
        st = L.mtlg_spmv_dot_noalloc(4, 4, *args, ok, None)
        assert st == _lib.ERR_INVALID_ARG, missing


def test_trace_report_api_without_gpu():
    from mtl4_b200 import trace
    trace.reset()
    trace.enable(True)
    assert trace.report() == {}
    trace.enable(False)


def test_server_admission_rule_without_gpu():
    from mtl4_b200 import _lib
    L = _lib.load()
    GiB = 1 << 30
    # with a byte budget
    assert L.mtlg_server_admission(3 * GiB, 6 * GiB, 10 * GiB, 0, 0) == 1
    assert L.mtlg_server_admission(5 * GiB, 6 * GiB, 10 * GiB, 0, 0) == 0    # waits for retirements
    assert L.mtlg_server_admission(11 * GiB, 0, 10 * GiB, 0, 0) == -1        # never fits
    # by free memory (simulated 8 GiB free, 1 GiB reserve)
    assert L.mtlg_server_admission(7 * GiB, 0, 0, 8 * GiB, GiB) == 1
    assert L.mtlg_server_admission(7 * GiB + 1, 0, 0, 8 * GiB, GiB) == -1
    assert L.mtlg_server_admission(9 * GiB, 4 * GiB, 0, 8 * GiB, GiB) == 0   # room once held requests retire
    assert L.mtlg_server_admission(12 * GiB, 4 * GiB, 0, 8 * GiB, GiB) == -1
    assert L.mtlg_server_admission(1, 0, 0, GiB // 2, GiB) == -1            # free memory below the reserve
