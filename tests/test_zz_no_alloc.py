"""The allocation-free entry point mtlg_spmv_dot_noalloc, for callers that
cannot allocate device memory (a fully reserved budget, a foreign memory
pool, a real-time loop where cudaMalloc may block).  It is checked against
the library's regular fused SpMV + dot (mtlg_spmv_dot) on the same inputs,
twice in a row, since every call reuses the same static scratch array.

The test itself allocates its buffers with torch; only the entry point under
test must not allocate.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from mtl4_b200 import problems as P
from test_oracle import spmv_rel_err

pytestmark = pytest.mark.gpu

MAX_ROWS = 4096 * 256


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a).astype(dtype)).cuda()


def _noalloc(L, torch, A, rp, ci, val, p, q, dot, stream=None):
    """One call; returns (status, device bytes that the call took)."""
    stream = stream or torch.cuda.current_stream()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    st = L.mtlg_spmv_dot_noalloc(A.n_rows, A.n_cols, C.c_void_p(rp.data_ptr()), C.c_void_p(ci.data_ptr()),
                                 C.c_void_p(val.data_ptr()), C.c_void_p(p.data_ptr()), C.c_void_p(q.data_ptr()),
                                 C.c_void_p(dot.data_ptr()), C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return st, free_before - torch.cuda.mem_get_info()[0]


@pytest.mark.parametrize("kind", ["stencil", "irregular"])
def test_noalloc_matches_regular_entry_point_twice(kind):
    torch = pytest.importorskip("torch")
    from mtl4_b200 import _lib, mtl
    L = _lib.lib()
    ctx = mtl.context(0)
    A = P.laplacian_2d(300) if kind == "stencil" else P.powerlaw_csr(200_000, seed=2)
    Ad = mtl.compressed2D.from_problem(A, ctx)
    rp = _dev(torch, A.row_ptr, np.int32)
    ci = _dev(torch, A.col, np.int32)
    val = _dev(torch, A.val, np.float64)
    rng = np.random.default_rng(17)
    # set-up call: the first call on a device looks up the scratch array's
    # address (and loads the module that holds it, which is where the array
    # itself lives); the calls checked below must take no device memory
    q0 = torch.zeros(A.n_rows, dtype=torch.float64, device="cuda")
    d0 = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert _noalloc(L, torch, A, rp, ci, val, q0, q0.clone(), d0)[0] == _lib.OK
    side = torch.cuda.Stream()
    for call in range(2):
        x = rng.standard_normal(A.n_rows)
        p = _dev(torch, x, np.float64)
        q = torch.full((A.n_rows,), 7.0, dtype=torch.float64, device="cuda")
        dot = torch.zeros(1, dtype=torch.float64, device="cuda")
        # the second call runs on another stream (after the first finished)
        st, taken = _noalloc(L, torch, A, rp, ci, val, p, q, dot, stream=side if call else None)
        assert st == _lib.OK, call
        assert taken == 0, (call, taken)
        # the regular entry point on the same inputs
        qd = mtl.dense_vector(A.n_rows, np.float64, ctx)
        d_ref = mtl.mult_dot(Ad, mtl.dense_vector(x, np.float64, ctx), qd)
        q_ref = qd.numpy()
        q_new = q.cpu().numpy()
        assert spmv_rel_err(A, x, q_new, q_ref).max() <= 1e-14, call
        short = np.diff(A.row_ptr) <= 32
        assert np.array_equal(q_new[short], q_ref[short]), call
        scale = float(np.abs(x) @ np.abs(q_ref))
        assert abs(float(dot.item()) - d_ref) <= 1e-12 * scale, (call, float(dot.item()), d_ref)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    from mtl4_b200 import _lib
    L = _lib.lib()
    t = torch.zeros(4, dtype=torch.float64, device="cuda")
    ptr = C.c_void_p(t.data_ptr())
    n = MAX_ROWS + 1
    st = L.mtlg_spmv_dot_noalloc(n, n, ptr, ptr, ptr, ptr, ptr, ptr, None)
    assert st == _lib.ERR_TOO_LARGE
    assert b"allocation-free limit" in L.mtlg_last_error_message()
