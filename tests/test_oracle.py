"""Pins the CPU oracle: the restatement (oracle/mtl_oracle.cpp) against the
known-answer vectors of MTL4's own tests, against the golden fixtures made by
the reference build, and -- where oracle/_ref is present -- against the
reference build directly.  No GPU."""
import numpy as np
import pytest

from conftest import csr_from
from mtl4_b200 import problems as P
from oracle import oracle as O


# ---------------------------------------------------------------- reference KATs
def test_kat_spmv_stencil_5x5():
    # libs/numeric/mtl/test/matrix_vector_product_test.cpp:56-89: 5x5-grid
    # Laplacian times its column 12 gives the stencil 20,-8,1,0,-8,2,1 and
    # doubles under +=, restores under -=.
    A = P.laplacian_2d(5)
    dense = A.to_scipy().toarray()
    v = dense[12].copy()
    w = O.port_spmv(A, v)
    assert (w[12], w[13], w[14], w[15], w[17], w[18], w[22]) == (20, -8, 1, 0, -8, 2, 1)
    w2 = O.port_spmv(A, v, assign=1, y=w)
    assert w2[12] == 40 and w2[18] == 4
    w3 = O.port_spmv(A, v, assign=2, y=w2)
    assert w3[12] == 20 and w3[18] == 2


def test_kat_ic0_golden_vector():
    # libs/numeric/itl/test/ic_0_test.cpp:20-36: ic_0<M,float> on the 3x3-grid
    # Laplacian, solve(P, iota(9)), within ||.|| < 1e-3
    A = P.laplacian_2d(3)
    y = O.port_pc_apply(A, "ic_0", np.arange(9.0), storage_f32=True)
    yc = np.array([1.03194, 1.60198, 1.45357, 2.5258, 3.55386, 3.16, 2.91787, 4.09338, 3.81335])
    assert np.linalg.norm(y - yc) < 1e-3


def test_kat_dot_285():
    # libs/numeric/mtl/test/dot_test.cpp:28-45
    v = np.arange(1.0, 10.0)
    assert O.port_lib().mtlo_dot(9, O._p(v), O._p(v)) == 285.0


def _upper_5x5():
    # libs/numeric/mtl/test/trisolve_test.cpp:20-27
    rows = {0: [(0, 7)], 1: [(1, 8), (3, 2), (4, 3)], 2: [(2, 2)], 3: [(3, 4)], 4: [(4, 9)]}
    rp, ci, v = [0], [], []
    for r in range(5):
        for c, val in rows[r]:
            ci.append(c); v.append(float(val))
        rp.append(len(ci))
    return P.CSR(5, 5, np.array(rp, np.int64), np.array(ci, np.int32), np.array(v))


def test_kat_trisolve_upper_and_lower_exact():
    # trisolve_test.cpp:29-61: x = 1..5 recovered by upper and lower solves.
    # ILU(0) of a triangular matrix is that matrix (L or U part trivial), so
    # solve(P, b) is exactly the triangular solve.
    U = _upper_5x5()
    x = np.arange(1.0, 6.0)
    b = U.to_scipy() @ x
    assert np.allclose(O.port_pc_apply(U, "ilu_0", b), x, atol=1e-12)
    Lt = U.to_scipy().T.tocsr()
    Lc = P.CSR(5, 5, Lt.indptr.astype(np.int64), Lt.indices.astype(np.int32), Lt.data.astype(np.float64))
    bl = Lt @ x
    assert np.allclose(O.port_pc_apply(Lc, "ilu_0", bl), x, atol=1e-12)


def test_kat_ilu0_matches_dense_ikj():
    # libs/numeric/itl/test/ilu_0_test.cpp:31-50: sparse ILU(0) entries equal a
    # dense IKJ elimination restricted to the pattern.
    rng = np.random.default_rng(5)
    n = 12
    M = np.eye(n)
    for _ in range(2 * n):
        r, c = rng.integers(0, n, 2)
        M[r, c] -= 1
        M[r, r] += 1
    import scipy.sparse as sp
    S = sp.csr_matrix(M)
    S.sort_indices()
    A = P.CSR(n, n, S.indptr.astype(np.int64), S.indices.astype(np.int32), S.data.astype(np.float64))
    LU = M.copy()
    for i in range(1, n):
        for k in range(i):
            if LU[i, k] == 0 or M[i, k] == 0:
                continue
            LU[i, k] /= LU[k, k]
            for j in range(k + 1, n):
                if M[i, j] != 0:
                    LU[i, j] -= LU[i, k] * LU[k, j]
    Lrp, Lci, Lv = O.port_factor(A, "ilu_0", "L")
    Urp, Uci, Uv = O.port_factor(A, "ilu_0", "U")
    for i in range(n):
        for e in range(Lrp[i], Lrp[i + 1]):
            assert abs(Lv[e] - LU[i, Lci[e]]) < 1e-12
        for e in range(Urp[i], Urp[i + 1]):
            want = 1.0 / LU[i, i] if Uci[e] == i else LU[i, Uci[e]]
            assert abs(Uv[e] - want) < 1e-12


# ---------------------------------------------------------------- golden fixtures
def test_laplacian_generator_matches_reference_setup(golden):
    A = P.laplacian_2d(32)
    assert np.array_equal(A.row_ptr, golden["lap32_rp"])
    assert np.array_equal(A.col, golden["lap32_ci"])
    assert np.array_equal(A.val, golden["lap32_val"])


def iterations_ok(solver, it, ref_it):
    """Equal or fewer iterations, +-2: at most the reference's count + 2 (CG
    also at least its count - 2).  The restatement, and the GPU in its
    reference summation order, take exactly the reference's count."""
    if solver == "cg":
        return abs(it - ref_it) <= 2
    return it <= ref_it + 2


def sha256(x):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(x, dtype=np.float64).tobytes()).hexdigest()


def spmv_rel_err(A, x, y, y_ref):
    """Per-entry error relative to sum_j |a_ij x_j| (the scale of row i)."""
    scale = P.CSR(A.n_rows, A.n_cols, A.row_ptr, A.col, np.abs(A.val)).matvec(np.abs(x).astype(np.float64))
    scale[scale == 0] = 1.0
    return np.abs(y.astype(np.float64) - y_ref.astype(np.float64)) / scale


def test_port_spmv_golden(golden):
    # stencil values: every product is exact, so the row sums are bitwise equal
    A = csr_from(golden, "lap32")
    assert np.array_equal(O.port_spmv(A, golden["lap32_x"]), golden["lap32_spmv"])
    assert np.array_equal(O.port_spmv(A, golden["lap32_x"].astype(np.float32)), golden["lap32_spmv_f32"])
    # general values: the reference build adds rounded products in groups of
    # four and fuses each row's last (L mod 4) FP64 steps; the restatement
    # follows that rule, so every row (up to 4096 entries here) is bitwise
    Q = csr_from(golden, "pl")
    x = golden["pl_x"]
    assert np.array_equal(O.port_spmv(Q, x), golden["pl_spmv"])
    assert np.array_equal(O.port_spmv(Q, x.astype(np.float32)), golden["pl_spmv_f32"])


@pytest.mark.parametrize("kind", ["ilu_0", "ic_0"])
def test_port_factors_bitwise_golden(golden, kind):
    A = csr_from(golden, "cd8")
    for which in "LU":
        rp, ci, v = O.port_factor(A, kind, which)
        assert np.array_equal(rp, golden[f"cd8_{kind}_{which}_rp"])
        assert np.array_equal(ci, golden[f"cd8_{kind}_{which}_ci"])
        assert np.array_equal(v, golden[f"cd8_{kind}_{which}_val"])


@pytest.mark.parametrize("kind", ["diagonal", "ilu_0", "ic_0"])
def test_port_apply_bitwise_golden(golden, kind):
    A = csr_from(golden, "cd8")
    x = golden["cd8_x"]
    assert np.array_equal(O.port_pc_apply(A, kind, x), golden[f"cd8_{kind}_apply_f64"])
    if kind != "diagonal":
        assert np.array_equal(O.port_pc_apply(A, kind, x, storage_f32=True), golden[f"cd8_{kind}_apply_f64s32"])
    assert np.array_equal(O.port_pc_apply(A, kind, x.astype(np.float32)), golden[f"cd8_{kind}_apply_f32"])


SOLVES = [("cg", "diagonal"), ("cg", "identity"), ("cg", "ic_0"), ("bicgstab", "ilu_0"), ("bicgstab", "diagonal"),
          ("bicgstab", "identity"), ("bicgstab", "ic_0")]


@pytest.mark.parametrize("solver,pc", SOLVES)
def test_port_solve_iterations_golden(golden, solver, pc):
    A = csr_from(golden, "lap32")
    r = O.port_solve(A, golden["lap32_b"], solver, pc, max_iter=2000, rtol=1e-8)
    ref_it = int(golden[f"lap32_{solver}_{pc}_iters"])
    assert r["error"] == 0
    # the restatement follows the reference build's arithmetic step by step
    # (contractions, summation orders): same count, bitwise the same x
    assert r["iterations"] == ref_it
    assert np.array_equal(r["x"], golden[f"lap32_{solver}_{pc}_x"])
    # the solution meets the residual tolerance (true residual, FP64) and
    # agrees with the reference's to the accuracy that tolerance implies
    b = golden["lap32_b"]
    assert np.linalg.norm(A.matvec(r["x"]) - b) <= 1.05e-8 * np.linalg.norm(b)
    assert np.abs(r["x"] - golden[f"lap32_{solver}_{pc}_x"]).max() < 1e-4


def test_port_dot_and_norm_in_reference_order(golden):
    L = O.port_lib()
    x, y = golden["dot_x"], golden["dot_y"]
    assert L.mtlo_dot4(x.size, O._p(x), O._p(y)) == float(golden["dot_xy"])
    assert np.sqrt(L.mtlo_norm4(x.size, O._p(x))) == float(golden["norm_x"])


@pytest.mark.parametrize("tag", ["c1", "c2"])
def test_port_full_size_solve_bitwise(golden, tag):
    # config 1 (CG + diagonal, 256^2) and config 2 (BiCGSTAB + ILU(0), 128^3):
    # the restatement's x is the reference build's x, byte for byte
    A, b, _ = P.config1() if tag == "c1" else P.config2_solve(128)
    solver, pc = ("cg", "diagonal") if tag == "c1" else ("bicgstab", "ilu_0")
    r = O.port_solve(A, b, solver, pc, max_iter=2000, rtol=1e-8)
    assert r["iterations"] == int(golden[f"{tag}_iters"])
    assert r["relresid"] == float(golden[f"{tag}_relres"])
    assert sha256(r["x"]) == str(golden[f"{tag}_x_sha256"])


def test_port_refinement_reaches_tolerance(golden):
    A = csr_from(golden, "lap32")
    b = golden["lap32_b"]
    r = O.port_refine(A, b, "cg", "ic_0", rtol=1e-10, inner_rtol=1e-4)
    assert r["error"] == 0 and r["relresid"] <= 1e-10
    xr = r["x"]
    assert np.linalg.norm(A.matvec(xr) - b) <= 1e-10 * np.linalg.norm(b) * 1.01


def test_port_gmres_restatement_converges():
    # libs/numeric/itl/test/gmres_test.cpp:52-128: 2x2-grid Laplacian,
    # GMRES(k) for k = 1..8 reaches ||r|| < 5e-5
    A = P.laplacian_2d(2)
    b = np.ones(4)
    for k in range(1, 9):
        r = O.port_solve(A, b, "gmres", "identity", max_iter=100, rtol=1e-10, restart=k)
        assert np.linalg.norm(A.matvec(r["x"]) - b) < 5e-5


# ---------------------------------------------------------------- reference build
@pytest.mark.ref
def test_reference_ilu0_adjoint_solves_the_transposed_system(need_ref):
    # adjoint_solve(P, x) of pc::ilu_0 (itl/pc/ilu.hpp:104-115): (L U)^T y = x
    # with L unit lower and U stored with its inverted diagonal
    import scipy.sparse as sp
    A, _, _ = P.config2_solve(6)
    R = need_ref.RefMatrix(A)
    (Lrp, Lci, Lv), (Urp, Uci, Uv) = R.factors("ilu_0")
    n = A.n_rows
    Ld = sp.csr_matrix((Lv, Lci, Lrp), shape=(n, n)).toarray()
    Ud = sp.csr_matrix((Uv, Uci, Urp), shape=(n, n)).toarray()
    Ld = Ld - np.diag(np.diag(Ld)) + np.eye(n)
    Ud = Ud - np.diag(np.diag(Ud)) + np.diag(1.0 / np.diag(Ud))
    x = np.random.default_rng(0).standard_normal(n)
    y = R.pc_adjoint_apply("ilu_0", x)
    assert np.abs((Ld @ Ud).T @ y - x).max() <= 1e-13 * np.abs(x).max() * n


@pytest.mark.ref
def test_port_equals_reference_build(need_ref):
    A = P.convdiff_3d(10)
    R = need_ref.RefMatrix(A)
    x = np.random.default_rng(3).standard_normal(A.n_rows)
    assert np.array_equal(O.port_spmv(A, x), R.spmv(x))
    y0 = np.random.default_rng(4).standard_normal(A.n_rows)
    for assign in (1, 2):
        assert np.array_equal(O.port_spmv(A, x, assign, y0), R.spmv(x, assign, y0))
    Q = P.powerlaw_csr(50_000, seed=7)
    xq = np.random.default_rng(5).standard_normal(Q.n_cols)
    RQ = need_ref.RefMatrix(Q)
    assert np.array_equal(O.port_spmv(Q, xq), RQ.spmv(xq))
    assert np.array_equal(O.port_spmv(Q, xq.astype(np.float32)), RQ.spmv(xq.astype(np.float32)))
    for kind in ["diagonal", "ilu_0", "ic_0"]:
        assert np.array_equal(R.pc_apply(kind, x), O.port_pc_apply(A, kind, x))
        assert np.array_equal(R.pc_apply(kind, x.astype(np.float32)), O.port_pc_apply(A, kind, x.astype(np.float32)))
    _, b = P.rhs_from_solution(A, 1)
    for solver, pc in SOLVES:
        a = R.solve(b, solver, pc)
        c = O.port_solve(A, b, solver, pc)
        assert c["iterations"] == a["iterations"] and np.array_equal(c["x"], a["x"]), (solver, pc)
