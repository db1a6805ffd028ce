"""GPU parity: the CUDA library (through its C ABI) against the oracle on the
same seeded inputs.  SpMV: bitwise on every row of up to 32 entries (the
oracle's row sum is bitwise the reference build's), <= 1e-14 relative per
entry (FP64) on longer rows, which a warp sums as a tree; factors and
preconditioner applies: bitwise; solves: the true FP64 residual meets the
tolerance and the iteration count is at most the reference's + 2."""
import numpy as np
import pytest

from conftest import csr_from
from mtl4_b200 import problems as P
from oracle import oracle as O
from test_oracle import iterations_ok, spmv_rel_err

pytestmark = pytest.mark.gpu


def dev(A, ctx):
    from mtl4_b200 import mtl
    return mtl.compressed2D.from_problem(A, ctx)


def vec(a, ctx, dtype=np.float64):
    from mtl4_b200 import mtl
    return mtl.dense_vector(np.asarray(a, dtype=dtype), dtype, ctx)


# ---------------------------------------------------------------- SpMV
def test_spmv_kat_stencil(ctx):
    from mtl4_b200 import mtl
    A = P.laplacian_2d(5)
    Ad = dev(A, ctx)
    v = vec(A.to_scipy().toarray()[12], ctx)
    w = mtl.dense_vector(25, np.float64, ctx)
    w.assign(Ad * v)
    h = w.numpy()
    assert (h[12], h[13], h[14], h[15], h[17], h[18], h[22]) == (20, -8, 1, 0, -8, 2, 1)
    w += Ad * v
    assert w.numpy()[12] == 40 and w.numpy()[18] == 4
    w -= Ad * v
    assert w.numpy()[12] == 20 and w.numpy()[18] == 2


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_spmv_stencil_bitwise(ctx, golden, dtype):
    from mtl4_b200 import mtl
    A = csr_from(golden, "lap32")
    Ad = dev(A, ctx)
    x = golden["lap32_x"].astype(dtype)
    y = mtl.dense_vector(A.n_rows, dtype, ctx)
    mtl.mult(Ad, vec(x, ctx, dtype), y)
    want = golden["lap32_spmv"] if dtype == np.float64 else golden["lap32_spmv_f32"]
    assert np.array_equal(y.numpy(), want)


@pytest.mark.parametrize("n", [5000, 200_000])
def test_spmv_irregular(ctx, n):
    from mtl4_b200 import mtl
    Q = P.powerlaw_csr(n, seed=2)
    Qd = dev(Q, ctx)
    x = np.random.default_rng(4).standard_normal(n)
    y = mtl.dense_vector(n, np.float64, ctx)
    mtl.mult(Qd, vec(x, ctx), y)
    ref = O.port_spmv(Q, x)
    err = spmv_rel_err(Q, x, y.numpy(), ref)
    assert err.max() <= 1e-14
    # rows of up to 32 entries keep the sequential order: bitwise
    short = np.diff(Q.row_ptr) <= 32
    assert np.array_equal(y.numpy()[short], ref[short])
    # += and -=
    y2 = vec(np.ones(n), ctx)
    mtl.mult(Qd, vec(x, ctx), y2, "-=")
    assert spmv_rel_err(Q, x, y2.numpy(), 1.0 - ref).max() <= 1e-14
    xf = x.astype(np.float32)
    yf = mtl.dense_vector(n, np.float32, ctx)
    mtl.mult(Qd, vec(xf, ctx, np.float32), yf)
    assert spmv_rel_err(Q, xf, yf.numpy(), O.port_spmv(Q, xf)).max() <= 1e-6


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_spmv_general_values_bitwise(ctx, dtype):
    # convection-diffusion values: products are not exact, so this pins the
    # reference's contraction rule (rounded groups of four, fused FP64 tail)
    # in the standalone SpMV and in the fused SpMV + dot of the solvers
    from mtl4_b200 import mtl
    A = P.convdiff_3d(20)
    Ad = dev(A, ctx)
    x = np.random.default_rng(6).uniform(-1, 1, A.n_rows).astype(dtype)
    y = mtl.dense_vector(A.n_rows, dtype, ctx)
    mtl.mult(Ad, vec(x, ctx, dtype), y)
    ref = O.port_spmv(A, x)
    assert np.array_equal(y.numpy(), ref)
    if dtype == np.float64:
        q = mtl.dense_vector(A.n_rows, dtype, ctx)
        mtl.mult_dot(Ad, vec(x, ctx, dtype), q)
        assert np.array_equal(q.numpy(), ref)


def test_spmv_long_rows_and_empty_rows(ctx):
    from mtl4_b200 import mtl
    # rows longer than a shared-memory tile, empty rows, a 1x1 and an empty matrix
    rng = np.random.default_rng(9)
    n = 6000
    lengths = np.zeros(n, np.int64)
    lengths[::7] = rng.integers(1, 40, len(lengths[::7]))
    lengths[100] = 5000
    lengths[4000] = 2049
    rp = np.concatenate([[0], np.cumsum(lengths)])
    ci = np.concatenate([np.sort(rng.choice(n, int(L), replace=False)) for L in lengths]).astype(np.int32)
    A = P.CSR(n, n, rp, ci, rng.standard_normal(int(rp[-1])))
    Ad = dev(A, ctx)
    assert Ad.plan_info()["long_tiles"] == 2
    x = rng.standard_normal(n)
    y = vec(np.full(n, 7.0), ctx)
    mtl.mult(Ad, vec(x, ctx), y)
    assert spmv_rel_err(A, x, y.numpy(), O.port_spmv(A, x)).max() <= 1e-14
    assert np.all(y.numpy()[lengths == 0] == 0.0)
    one = P.CSR(1, 1, np.array([0, 1], np.int64), np.array([0], np.int32), np.array([3.0]))
    y1 = vec([0.0], ctx)
    mtl.mult(dev(one, ctx), vec([2.0], ctx), y1)
    assert y1.numpy()[0] == 6.0


def test_spmv_dot_fused(ctx):
    from mtl4_b200 import mtl
    # (lazy(w) = B * v) || (lazy(d) = lazy_dot(w, v)) with B all 2, v all 1
    # (libs/numeric/mtl/test/fuse_test.cpp)
    n = 6
    rp = np.arange(0, n * n + 1, n, dtype=np.int64)
    ci = np.tile(np.arange(n, dtype=np.int32), n)
    B = P.CSR(n, n, rp, ci, np.full(n * n, 2.0))
    q = mtl.dense_vector(n, np.float64, ctx)
    d = mtl.mult_dot(dev(B, ctx), vec(np.ones(n), ctx), q)
    assert np.all(q.numpy() == 12.0) and d == 72.0


def test_dot_norm_axpy(ctx):
    from mtl4_b200 import mtl
    a = vec(np.arange(1.0, 10.0), ctx)
    assert mtl.dot(a, a) == 285.0                       # dot_test.cpp:38-44
    assert abs(mtl.two_norm(a) - np.sqrt(285.0)) < 1e-14
    x = np.random.default_rng(1).standard_normal(100_003)
    xd, yd = vec(x, ctx), vec(np.ones_like(x), ctx)
    assert abs(mtl.dot(xd, yd) - x.sum()) <= 1e-12 * np.abs(x).sum()
    mtl.axpy(2.0, xd, yd)
    assert np.allclose(yd.numpy(), 1.0 + 2.0 * x, rtol=0, atol=1e-15)


def test_errors_map_to_reference_exceptions(ctx):
    from mtl4_b200 import _lib, itl, mtl
    A = P.laplacian_2d(4)
    Ad = dev(A, ctx)
    with pytest.raises(_lib.incompatible_size):
        mtl.mult(Ad, vec(np.ones(3), ctx), vec(np.ones(16), ctx))
    rect = mtl.compressed2D(np.array([0, 1, 2]), np.array([0, 1]), np.ones(2), shape=(2, 3), ctx=ctx)
    with pytest.raises(_lib.matrix_not_square):
        itl.pc.ilu_0(rect)
    nodiag = P.CSR(2, 2, np.array([0, 1, 2], np.int64), np.array([1, 0], np.int32), np.ones(2))
    with pytest.raises(_lib.missing_diagonal):
        itl.pc.ic_0(dev(nodiag, ctx))
    with pytest.raises(_lib.logic_error):
        mtl.compressed2D(np.array([0, 2]), np.array([1, 0]), np.ones(2), ctx=ctx)   # unsorted row


# ---------------------------------------------------------------- preconditioners
@pytest.mark.parametrize("kind", ["ilu_0", "ic_0"])
def test_factors_bitwise(ctx, golden, kind):
    from mtl4_b200 import itl
    A = csr_from(golden, "cd8")
    Pc = getattr(itl.pc, kind)(dev(A, ctx))
    for which in "LU":
        rp, ci, v = Pc.factor(which)
        assert np.array_equal(rp, golden[f"cd8_{kind}_{which}_rp"])
        assert np.array_equal(ci, golden[f"cd8_{kind}_{which}_ci"])
        assert np.array_equal(v, golden[f"cd8_{kind}_{which}_val"])


@pytest.mark.parametrize("kind", ["diagonal", "ilu_0", "ic_0"])
@pytest.mark.parametrize("mode", ["f64", "f64s32", "f32"])
def test_pc_apply_bitwise(ctx, golden, kind, mode):
    from mtl4_b200 import itl
    if kind == "diagonal" and mode == "f64s32":
        pytest.skip("the reference has solve() only for diagonal<Matrix> in the matrix's type")
    A = csr_from(golden, "cd8")
    storage = np.float32 if mode in ("f64s32", "f32") else np.float64
    Pc = getattr(itl.pc, kind)(dev(A, ctx), storage)
    vt = np.float32 if mode == "f32" else np.float64
    y = itl.solve(Pc, vec(golden["cd8_x"].astype(vt), ctx, vt))
    assert np.array_equal(y.numpy(), golden[f"cd8_{kind}_apply_{mode}"])


@pytest.mark.parametrize("m", [48, 160])
def test_sweeps_large_grid_match_restatement(ctx, m):
    from mtl4_b200 import itl
    A = P.vardiff_2d(m, sigma=1.0, seed=7)
    Ad = dev(A, ctx)
    x = np.random.default_rng(2).standard_normal(A.n_rows)
    for kind in ["ilu_0", "ic_0"]:
        Pc = getattr(itl.pc, kind)(Ad)
        assert Pc.levels()[0] == 2 * m - 1
        y = itl.solve(Pc, vec(x, ctx))
        assert np.array_equal(y.numpy(), O.port_pc_apply(A, kind, x))


def test_ic0_golden_vector(ctx):
    from mtl4_b200 import itl
    # libs/numeric/itl/test/ic_0_test.cpp:20-36
    A = P.laplacian_2d(3)
    Pc = itl.pc.ic_0(dev(A, ctx), np.float32)
    y = itl.solve(Pc, vec(np.arange(9.0), ctx)).numpy()
    yc = np.array([1.03194, 1.60198, 1.45357, 2.5258, 3.55386, 3.16, 2.91787, 4.09338, 3.81335])
    assert np.linalg.norm(y - yc) < 1e-3


def test_trisolve_kat_exact(ctx):
    from mtl4_b200 import itl
    from test_oracle import _upper_5x5
    U = _upper_5x5()
    x = np.arange(1.0, 6.0)
    y = itl.solve(itl.pc.ilu_0(dev(U, ctx)), vec(U.to_scipy() @ x, ctx)).numpy()
    assert np.allclose(y, x, atol=1e-12)


# ---------------------------------------------------------------- solvers
def solve_gpu(ctx, A, b, solver, pc, rtol=1e-8, max_iter=2000, storage=np.float64, dtype=np.float64):
    from mtl4_b200 import itl, mtl
    Ad = dev(A, ctx)
    Pc = None if pc == "identity" else getattr(itl.pc, pc)(Ad, storage)
    x = mtl.dense_vector(A.n_rows, dtype, ctx)
    bd = vec(b, ctx, dtype)
    it = itl.basic_iteration(bd, max_iter, rtol)
    getattr(itl, solver)(Ad, x, bd, Pc, it)
    return x.numpy(), it


@pytest.mark.parametrize("solver,pc", [("cg", "diagonal"), ("cg", "identity"), ("cg", "ic_0"),
                                       ("bicgstab", "ilu_0"), ("bicgstab", "diagonal"), ("bicgstab", "identity")])
def test_solve_lap32(ctx, golden, solver, pc):
    A = csr_from(golden, "lap32")
    b = golden["lap32_b"]
    x, it = solve_gpu(ctx, A, b, solver, pc)
    ref_key = f"lap32_{solver}_{pc}_iters"
    ref_it = int(golden[ref_key]) if ref_key in golden else O.port_solve(A, b, solver, pc)["iterations"]
    assert it.error_code() == 0 and it.is_converged()
    assert iterations_ok(solver, it.iterations(), ref_it), (it.iterations(), ref_it)
    assert np.linalg.norm(A.matvec(x) - b) <= 1.05e-8 * np.linalg.norm(b)


def test_cg_config1_laplacian_256(ctx):
    A, b, _ = P.config1()
    x, it = solve_gpu(ctx, A, b, "cg", "diagonal")
    ref = O.port_solve(A, b, "cg", "diagonal", max_iter=2000, rtol=1e-8)
    assert it.is_converged() and abs(it.iterations() - ref["iterations"]) <= 2
    assert np.linalg.norm(A.matvec(x) - b) <= 1.05e-8 * np.linalg.norm(b)


def test_bicgstab_ilu0_convdiff(ctx):
    A, b, _ = P.config2_solve(24)
    x, it = solve_gpu(ctx, A, b, "bicgstab", "ilu_0")
    ref = O.port_solve(A, b, "bicgstab", "ilu_0", max_iter=2000, rtol=1e-8)
    assert it.is_converged() and iterations_ok("bicgstab", it.iterations(), ref["iterations"])
    assert np.linalg.norm(A.matvec(x) - b) <= 1.05e-8 * np.linalg.norm(b)


def test_max_iterations_reports_error_1(ctx):
    A, b, _ = P.config1()
    x, it = solve_gpu(ctx, A, b, "cg", "diagonal", max_iter=7)
    assert it.error_code() == 1 and it.iterations() == 7 and not it.is_converged()


def test_zero_rhs_converges_immediately(ctx):
    A = P.laplacian_2d(16)
    x, it = solve_gpu(ctx, A, np.zeros(A.n_rows), "cg", "ic_0")
    assert it.iterations() == 0 and np.all(x == 0)


def test_solver_reuse_same_operator(ctx):
    # the loop graph is built once per (operator, preconditioner) and reused
    from mtl4_b200 import itl, mtl
    A = P.laplacian_2d(40)
    Ad = dev(A, ctx)
    Pc = itl.pc.ic_0(Ad)
    for seed in range(3):
        _, b = P.rhs_from_solution(A, seed)
        x = mtl.dense_vector(A.n_rows, np.float64, ctx)
        bd = vec(b, ctx)
        it = itl.basic_iteration(bd, 500, 1e-8)
        itl.cg(Ad, x, bd, Pc, it)
        assert it.is_converged()
        assert np.linalg.norm(A.matvec(x.numpy()) - b) <= 1.05e-8 * np.linalg.norm(b)


# ---------------------------------------------------------------- mixed precision
@pytest.mark.parametrize("solver,pc", [("cg", "ic_0"), ("cg", "diagonal"), ("bicgstab", "ilu_0")])
def test_refinement_fp32_inner_fp64_outer(ctx, solver, pc):
    from mtl4_b200 import itl, mtl
    A = P.vardiff_2d(64, sigma=1.0, seed=3) if solver == "cg" else P.convdiff_3d(16)
    _, b = P.rhs_from_solution(A, 3)
    Ad = dev(A, ctx)
    Pc = getattr(itl.pc, pc)(Ad, np.float32)
    x = mtl.dense_vector(A.n_rows, np.float64, ctx)
    it = itl.refine(solver, Ad, x, vec(b, ctx), Pc, rtol=1e-10, inner_rtol=1e-4)
    assert it.is_converged() and it.outer >= 1
    xs = x.numpy()
    rel = np.linalg.norm(A.matvec(xs) - b) / np.linalg.norm(b)
    assert rel <= 1e-10
    x64 = O.port_solve(A, b, solver, pc, max_iter=5000, rtol=1e-13)["x"]
    assert np.abs(xs - x64).max() <= 1e-6 * np.abs(x64).max()
    assert not it.fp64_fallback


def ill_conditioned_request():
    """A request of the served stream whose operator is too ill-conditioned
    for an FP32 inner solve (2D, 552^2, log-normal coefficients sigma = 1,
    weak convection): the FP32 BiCGSTAB + ILU(0) refinement does not reduce
    the FP64 residual."""
    sp = P.request_specs(20000)[33]
    assert (sp.dims, sp.m, sp.solver, sp.pc) == (2, 552, "bicgstab", "ilu_0")
    A = sp.build()
    return sp, A, P.random_rhs(A.n_rows, sp.seed)


def test_refinement_stall_finishes_in_fp64(ctx):
    from mtl4_b200 import itl, mtl
    sp, A, b = ill_conditioned_request()
    Ad = dev(A, ctx)
    x = mtl.dense_vector(A.n_rows, np.float64, ctx)
    it = itl.refine("bicgstab", Ad, x, vec(b, ctx), itl.pc.ilu_0(Ad, np.float32), rtol=1e-8, inner_rtol=1e-4)
    assert it.fp64_fallback and it.is_converged()
    rel = np.linalg.norm(A.matvec(x.numpy()) - b) / np.linalg.norm(b)
    assert rel <= 1e-8


# ---------------------------------------------------------------- GMRES
def test_gmres_kat_small_laplacian(ctx):
    # libs/numeric/itl/test/gmres_test.cpp:52-128: 2x2-grid Laplacian,
    # GMRES(k) for k = 1..8 reaches ||r|| < 5e-5
    from mtl4_b200 import itl, mtl
    A = P.laplacian_2d(2)
    Ad = dev(A, ctx)
    b = np.ones(4)
    for k in range(1, 9):
        x = mtl.dense_vector(4, np.float64, ctx)
        bd = vec(b, ctx)
        it = itl.basic_iteration(bd, 100, 1e-10)
        itl.gmres(Ad, x, bd, None, None, it, k)
        assert np.linalg.norm(A.matvec(x.numpy()) - b) < 5e-5


@pytest.mark.parametrize("restart,pc", [(10, "identity"), (30, "identity"), (20, "ilu_0"), (8, "diagonal")])
def test_gmres_matches_restatement(ctx, golden, restart, pc):
    from mtl4_b200 import itl, mtl
    A = csr_from(golden, "lap32")
    b = golden["lap32_b"]
    Ad = dev(A, ctx)
    L = None if pc == "identity" else getattr(itl.pc, pc)(Ad)
    x = mtl.dense_vector(A.n_rows, np.float64, ctx)
    bd = vec(b, ctx)
    it = itl.basic_iteration(bd, 3000, 1e-8)
    itl.gmres(Ad, x, bd, L, None, it, restart)
    ref = O.port_solve(A, b, "gmres", pc, max_iter=3000, rtol=1e-8, restart=restart)
    assert it.error_code() == ref["error"] == 0
    assert abs(it.iterations() - ref["iterations"]) <= restart   # same number of restart cycles (+-1)
    # a cycle may stop on the left-preconditioned residual ||L^-1 r||, as the
    # reference does (gmres.hpp:52-53); the true residual is within cond(L)
    assert it.resid() <= 1.05e-8 * np.linalg.norm(b)
    true = np.linalg.norm(A.matvec(x.numpy()) - b)
    assert true <= (1.05e-8 if pc == "identity" else 1e-7) * np.linalg.norm(b)


def test_gmres_max_iterations(ctx):
    from mtl4_b200 import itl, mtl
    A, b, _ = P.config1()
    Ad = dev(A, ctx)
    x = mtl.dense_vector(A.n_rows, np.float64, ctx)
    bd = vec(b, ctx)
    it = itl.basic_iteration(bd, 25, 1e-8)
    itl.gmres(Ad, x, bd, None, None, it, 10)
    assert it.error_code() == 1 and it.iterations() == 25


def test_trace_hooks_record_reference_event_ids(ctx):
    # the reference's vampir_trace ids: 7004 bicgstab, 5038 ilu_0::factorize,
    # 5039 ilu_0::solve (interface/vpt.cpp)
    from mtl4_b200 import trace
    trace.reset()
    trace.enable(True)
    try:
        A, b, _ = P.config2_solve(12)
        solve_gpu(ctx, A, b, "bicgstab", "ilu_0")
    finally:
        trace.enable(False)
    rep = trace.report()
    assert rep[7004][0] == "bicgstab" and rep[7004][1] == 1
    assert rep[5038][0] == "ilu_0::factorize" and rep[5038][2] > 0
    assert 9102 in rep and 9104 in rep   # set-up phases


def test_matrix_market_to_device_csr(ctx, tmp_path):
    # a symmetric-storage file (lower triangle) read straight into device CSR:
    # the same operator as the generator's, SpMV bitwise the oracle's and CG
    # + IC(0) on it as on the generated matrix
    from mtl4_b200 import itl, mtl
    A = P.vardiff_2d(40, sigma=0.5, seed=9)
    f = tmp_path / "vd.mtx"
    with open(f, "w") as fh:
        lower = [(i, int(A.col[e]), float(A.val[e])) for i in range(A.n_rows)
                 for e in range(A.row_ptr[i], A.row_ptr[i + 1]) if A.col[e] <= i]
        fh.write("%%MatrixMarket matrix coordinate real symmetric\n% vardiff 40x40\n")
        fh.write(f"{A.n_rows} {A.n_cols} {len(lower)}\n")
        for i, j, v in lower:
            fh.write(f"{i + 1} {j + 1} {v!r}\n")
    Ad = mtl.compressed2D.from_matrix_market(f, ctx)
    assert Ad.shape == (A.n_rows, A.n_cols) and Ad.nnz == A.nnz
    x = np.random.default_rng(8).standard_normal(A.n_rows)
    y = mtl.dense_vector(A.n_rows, np.float64, ctx)
    mtl.mult(Ad, vec(x, ctx), y)
    assert np.array_equal(y.numpy(), O.port_spmv(A, x))
    _, b = P.rhs_from_solution(A, 2)
    xs, it = solve_gpu(ctx, A, b, "cg", "ic_0")
    xm = mtl.dense_vector(A.n_rows, np.float64, ctx)
    Pm = itl.pc.ic_0(Ad)
    itm = itl.basic_iteration(vec(b, ctx), 2000, 1e-8)
    itl.cg(Ad, xm, vec(b, ctx), Pm, itm)
    assert itm.iterations() == it.iterations() and np.array_equal(xm.numpy(), xs)
