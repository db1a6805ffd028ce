"""Mixed precision at the full config-3 sizes: FP32 CSR values and vectors,
an FP32-stored IC(0) (factorized in FP64, as ic_0<M, float> does,
itl/pc/ic_0.hpp:124-130) inside FP64 iterative refinement to a relative
residual <= 1e-10, on

  3a: the 2048 x 2048 5-point Laplacian (4,194,304 unknowns, 20,963,328 nnz)
  3b: the 160^3 SPD 7-point diffusion operator with log-normal coefficients
      (sigma 1.0, seed 3; 4,096,000 unknowns, 28,518,400 nnz).

The FP64 oracle solve is the GPU's plain FP64 CG + IC(0) in the reference
summation order (reduction_order 1), whose arithmetic is the reference
build's step for step (bitwise at configs 1 and 2, tests/test_gpu_parity.py),
run to 1e-12."""
import numpy as np
import pytest

from mtl4_b200 import problems as P

pytestmark = pytest.mark.gpu

SIZES = {"3a": (4_194_304, 20_963_328), "3b": (4_096_000, 28_518_400)}


@pytest.mark.parametrize("which", ["3a", "3b"])
def test_config3_fp32_inner_fp64_refinement(ctx, which):
    from mtl4_b200 import itl, mtl
    A, b, x_true = P.config3a() if which == "3a" else P.config3b()
    assert (A.n_rows, A.nnz) == SIZES[which]
    Ad = mtl.compressed2D.from_problem(A, ctx)
    bd = mtl.dense_vector(b, np.float64, ctx)
    nb = np.linalg.norm(b)

    P32 = itl.pc.ic_0(Ad, np.float32)
    x = mtl.dense_vector(A.n_rows, np.float64, ctx)
    it = itl.refine("cg", Ad, x, bd, P32, rtol=1e-10, inner_rtol=1e-4, max_outer=40, max_inner=5000)
    xm = x.numpy()
    assert it.is_converged() and not it.fp64_fallback, (it.error_code(), it.outer, it.relresid())
    assert it.outer >= 2   # FP32 alone cannot reach 1e-10: refinement did work
    rm = np.linalg.norm(A.matvec(xm) - b)
    assert rm <= 1.01e-10 * nb, rm / nb

    ctx.set_tuning("reduction_order", 1)
    try:
        P64 = itl.pc.ic_0(Ad, np.float64)
        x64 = mtl.dense_vector(A.n_rows, np.float64, ctx)
        it64 = itl.basic_iteration(bd, 20000, 1e-12)
        itl.cg(Ad, x64, bd, P64, it64)
    finally:
        ctx.set_tuning("reduction_order", 0)
    assert it64.is_converged(), (it64.iterations(), it64.relresid())
    xr = x64.numpy()
    r64 = np.linalg.norm(A.matvec(xr) - b)
    assert r64 <= 1.01e-12 * nb
    # the two solutions differ by no more than their residuals allow
    assert np.linalg.norm(A.matvec(xm - xr)) <= 1.01e-10 * nb + r64
    err = np.abs(xm - xr).max() / np.abs(xr).max()
    print(f"config {which}: inner {it.iterations()} outer {it.outer} relres {rm / nb:.3e}; "
          f"FP64 oracle {it64.iterations()} iterations; max error vs oracle {err:.3e}; "
          f"vs x_true {np.abs(xm - x_true).max() / np.abs(x_true).max():.3e}")
