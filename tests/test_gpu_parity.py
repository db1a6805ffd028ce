"""GPU parity in the reference summation order (context tuning
"reduction_order" 1): FP64 dots, norms and the CG / BiCGSTAB solves follow
the reference build's arithmetic step by step -- the SpMV row sums, the
vector updates' contractions and the four strided partial sums of mtl::dot,
two_norm and the fused lazy dots -- so iteration counts are the reference's
and the solutions are bitwise the reference's.  The fixtures come from the
reference build (tests/golden/make_golden.py); at the full config sizes the
solution is compared through the SHA-256 of its bytes.

The default mode sums dots tile by tile (parallel, deterministic, another
order); its iteration counts are held to the reference's + 2."""
import hashlib

import numpy as np
import pytest

from conftest import csr_from
from mtl4_b200 import problems as P
from test_oracle import SOLVES, iterations_ok

pytestmark = pytest.mark.gpu


@pytest.fixture
def rctx(ctx):
    ctx.set_tuning("reduction_order", 1)
    yield ctx
    ctx.set_tuning("reduction_order", 0)


def sha256(x):
    return hashlib.sha256(np.ascontiguousarray(x, dtype=np.float64).tobytes()).hexdigest()


def solve(ctx, A, b, solver, pc, max_iter=2000, rtol=1e-8):
    from mtl4_b200 import itl, mtl
    Ad = mtl.compressed2D.from_problem(A, ctx)
    Pc = None if pc == "identity" else getattr(itl.pc, pc)(Ad, np.float64)
    x = mtl.dense_vector(A.n_rows, np.float64, ctx)
    bd = mtl.dense_vector(np.asarray(b, np.float64), np.float64, ctx)
    it = itl.basic_iteration(bd, max_iter, rtol)
    getattr(itl, solver)(Ad, x, bd, Pc, it)
    return x.numpy(), it


def ldot4(a, b):
    """lazy_dot of a fused expression: rounded products, four strided partial
    sums, ((t0 + t1) + t2) + t3 (numpy float64 reproduces it exactly)."""
    n = a.size
    nb = n // 4 * 4
    t = np.zeros(4)
    for i in range(0, nb, 4):
        t = t + a[i:i + 4] * b[i:i + 4]
    for i in range(nb, n):
        t[0] = t[0] + a[i] * b[i]
    return ((t[0] + t[1]) + t[2]) + t[3]


def test_dot_norm_and_fused_dot_in_reference_order(rctx, golden):
    from mtl4_b200 import mtl
    x = mtl.dense_vector(golden["dot_x"], np.float64, rctx)
    y = mtl.dense_vector(golden["dot_y"], np.float64, rctx)
    assert mtl.dot(x, y) == float(golden["dot_xy"])
    assert mtl.two_norm(x) == float(golden["norm_x"])
    A = csr_from(golden, "lap32")
    Ad = mtl.compressed2D.from_problem(A, rctx)
    p = golden["lap32_x"]
    q = mtl.dense_vector(A.n_rows, np.float64, rctx)
    pq = mtl.mult_dot(Ad, mtl.dense_vector(p, np.float64, rctx), q)
    assert np.array_equal(q.numpy(), golden["lap32_spmv"])
    assert pq == ldot4(p, golden["lap32_spmv"])


@pytest.mark.parametrize("solver,pc", SOLVES)
def test_lap32_solves_bitwise(rctx, golden, solver, pc):
    A = csr_from(golden, "lap32")
    x, it = solve(rctx, A, golden["lap32_b"], solver, pc)
    assert it.error_code() == 0
    assert it.iterations() == int(golden[f"lap32_{solver}_{pc}_iters"])
    assert np.array_equal(x, golden[f"lap32_{solver}_{pc}_x"])


def test_config1_cg_diagonal_bitwise(rctx, golden):
    A, b, _ = P.config1()
    x, it = solve(rctx, A, b, "cg", "diagonal")
    assert it.iterations() == int(golden["c1_iters"]) == 565
    assert it.relresid() == float(golden["c1_relres"])
    assert sha256(x) == str(golden["c1_x_sha256"])


def test_config2_bicgstab_ilu0_128_bitwise(rctx, golden):
    # BiCGSTAB + ILU(0) on the 128^3 convection-diffusion operator (2,097,152
    # unknowns): the reference's 68 iterations and its x, byte for byte
    A, b, _ = P.config2_solve(128)
    x, it = solve(rctx, A, b, "bicgstab", "ilu_0")
    assert it.iterations() == int(golden["c2_iters"]) == 68
    assert it.relresid() == float(golden["c2_relres"])
    assert sha256(x) == str(golden["c2_x_sha256"])


def test_config2_bicgstab_ilu0_128_default_order(ctx, golden):
    # the default (tile-parallel) summation order: at most the reference's
    # count + 2 at the full size, true FP64 residual within the tolerance
    A, b, _ = P.config2_solve(128)
    x, it = solve(ctx, A, b, "bicgstab", "ilu_0")
    assert it.is_converged()
    assert iterations_ok("bicgstab", it.iterations(), int(golden["c2_iters"])), it.iterations()
    assert np.linalg.norm(A.matvec(x) - b) <= 1.05e-8 * np.linalg.norm(b)


def test_config1_cg_diagonal_default_order(ctx, golden):
    A, b, _ = P.config1()
    x, it = solve(ctx, A, b, "cg", "diagonal")
    assert it.is_converged()
    assert iterations_ok("cg", it.iterations(), int(golden["c1_iters"])), it.iterations()
    assert np.linalg.norm(A.matvec(x) - b) <= 1.05e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("solver,pc,cycle,multi", [("cg", "diagonal", 10, 0), ("bicgstab", "ilu_0", 1, 0),
                                                   ("bicgstab", "identity", 5, 1)])
def test_cyclic_iteration_prints_the_reference_lines(rctx, golden, solver, pc, cycle, multi):
    # itl::cyclic_iteration / noisy_iteration: the device-side termination
    # tests are logged and replayed through finished(); in the reference
    # summation order the printed lines (residuals at 6 digits, the final
    # summary) are the reference build's, character for character
    import io
    from mtl4_b200 import itl, mtl
    A = csr_from(golden, "lap32")
    Ad = mtl.compressed2D.from_problem(A, rctx)
    Pc = None if pc == "identity" else getattr(itl.pc, pc)(Ad, np.float64)
    x = mtl.dense_vector(A.n_rows, np.float64, rctx)
    bd = mtl.dense_vector(golden["lap32_b"], np.float64, rctx)
    out = io.StringIO()
    if cycle == 1:
        it = itl.noisy_iteration(bd, 2000, 1e-8, out=out)
    else:
        it = itl.cyclic_iteration(bd, 2000, 1e-8, cycle=cycle, out=out)
    it.set_multi_print(bool(multi))
    getattr(itl, solver)(Ad, x, bd, Pc, it)
    assert out.getvalue() == str(golden[f"lap32_{solver}_{pc}_cyclic{cycle}_{multi}"])
