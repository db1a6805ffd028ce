"""GPU parity of the grid sweeps (factors whose pattern is a 5- or 7-point
grid stencil: x-lines per lane, planes or y-blocks per warp, rings between
warps, receiver warps between CTAs): preconditioner applies equal the
oracle's bit for bit for 2D and 3D grids whose sides are and are not
multiples of the warp and tile sizes, for ILU(0) and IC(0), in every
precision combination, with 4 and 8 compute warps; other patterns keep the
chunked sweeps; solves and batches (Jacobi and IC(0) systems mixed) give the
chunked kernel's results exactly; expired waits report a timeout and the
next apply is exact again."""
import contextlib

import numpy as np
import pytest

from mtl4_b200 import problems as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def tuning(ctx, **kv):
    old = {k: ctx.get_tuning(k) for k in kv}
    try:
        for k, v in kv.items():
            ctx.set_tuning(k, v)
        yield
    finally:
        for k, v in old.items():
            ctx.set_tuning(k, v)


def dev(A, ctx):
    from mtl4_b200 import mtl
    return mtl.compressed2D.from_problem(A, ctx)


def vec(a, ctx, dtype=np.float64):
    from mtl4_b200 import mtl
    return mtl.dense_vector(np.asarray(a, dtype=dtype), dtype, ctx)


GRIDS = {
    # 3D: y-blocks of 32 and partial ones, plane counts not a multiple of the tile,
    # lines long enough for blocks where every lane has a row
    "convdiff3d_20": lambda: P.convdiff_3d(20),
    "convdiff3d_72x40x20": lambda: P.vardiff_3d((72, 40, 20), sigma=0.3, seed=2, beta=(0.4, 0.2, 0.1)),
    "vardiff3d_33x40x13": lambda: P.vardiff_3d((33, 40, 13), sigma=1.0, seed=4, beta=(0.3, 0.2, 0.1)),
    "vardiff3d_7x70x9": lambda: P.vardiff_3d((7, 70, 9), sigma=0.5, seed=6),
    # 2D: several y-blocks per tile, a partial last block
    "vardiff2d_96": lambda: P.vardiff_2d(96, sigma=1.0, seed=7),
    "vardiff2d_50x300": lambda: P.vardiff_2d((50, 300), sigma=1.0, seed=8, beta=(0.2, 0.1)),
    "laplacian2d_31": lambda: P.laplacian_2d(31),
}

MODES = (("f64", np.float64, np.float64), ("f64s32", np.float64, np.float32),
         ("f32", np.float32, np.float32), ("f32s64", np.float32, np.float64))


def oracle_apply(A, kind, x, vt, st):
    if vt == np.float32 and st == np.float32:
        return O.port_pc_apply(A, kind, x.astype(np.float32))
    if vt == np.float64:
        return O.port_pc_apply(A, kind, x, storage_f32=(st == np.float32))
    return None   # FP32 vectors with FP64 factors: compared with the chunked kernel


@pytest.mark.parametrize("name", list(GRIDS))
@pytest.mark.parametrize("warps", [4, 8])
def test_grid_apply_matches_oracle(ctx, name, warps):
    from mtl4_b200 import itl
    A = GRIDS[name]()
    x = np.random.default_rng(5).standard_normal(A.n_rows)
    Ad = dev(A, ctx)
    with tuning(ctx, grid_warps=warps):
        for kind in ("ilu_0", "ic_0"):
            for mode, vt, st in MODES:
                Pc = getattr(itl.pc, kind)(Ad, st)
                plan = Pc.sweep_plan(vt)
                # the context's warp count where its shared memory fits, else four
                assert plan["kernel"] == "grid" and plan["threads"] in (128, 32 * warps), (name, plan)
                want = oracle_apply(A, kind, x, vt, st)
                if want is None:
                    with tuning(ctx, grid_sweep=0):
                        Pk = getattr(itl.pc, kind)(Ad, st)
                        want = itl.solve(Pk, vec(x.astype(vt), ctx, vt)).numpy()
                for _ in range(2):   # rings, tickets and reset vectors come back to their start state
                    y = itl.solve(Pc, vec(x.astype(vt), ctx, vt)).numpy()
                    assert np.array_equal(y, want), (name, kind, mode, warps)


def test_non_grid_patterns_keep_the_chunked_sweep(ctx):
    from mtl4_b200 import itl
    from test_gpu_sweep_chunks import paired_blocks, random_banded_spd
    for A in (random_banded_spd(3000), paired_blocks(2001)):
        Pc = itl.pc.ilu_0(dev(A, ctx))
        assert Pc.sweep_plan(np.float64)["kernel"] == "chunked"
        x = np.random.default_rng(2).standard_normal(A.n_rows)
        assert np.array_equal(itl.solve(Pc, vec(x, ctx)).numpy(), O.port_pc_apply(A, "ilu_0", x))


@pytest.mark.parametrize("solver,kind", [("cg", "ic_0"), ("bicgstab", "ilu_0")])
def test_grid_solve_equals_chunked_solve(ctx, solver, kind):
    # same applies bit for bit, hence the same iterations and x
    from mtl4_b200 import itl, mtl
    A = P.vardiff_3d(24, sigma=1.0, seed=5, beta=(0.05, 0.02, 0.01))
    b = np.random.default_rng(3).standard_normal(A.n_rows)
    Ad = dev(A, ctx)
    out = []
    for grid in (1, 0):
        with tuning(ctx, grid_sweep=grid):
            Pc = getattr(itl.pc, kind)(Ad)
            assert Pc.sweep_plan(np.float64)["kernel"] == ("grid" if grid else "chunked")
            x = mtl.dense_vector(A.n_rows, np.float64, ctx)
            bd = vec(b, ctx)
            it = itl.basic_iteration(bd, 1000, 1e-10)
            getattr(itl, solver)(Ad, x, bd, Pc, it)
            out.append((it.iterations(), x.numpy()))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("mixed", [False, True])
def test_grid_batch_with_jacobi_and_ic0_matches_standalone(ctx, mixed):
    # 2D and 3D systems with IC(0) and with Jacobi (trivial factors: an
    # unskewed grid of independent rows) in one set of grid sweeps
    from mtl4_b200 import serve
    probs = [P.vardiff_3d(m, sigma=0.5, seed=m) for m in (9, 14)] + \
            [P.vardiff_2d(m, sigma=0.5, seed=m) for m in (40, 75)]
    kinds = ["ic_0", "diagonal", "diagonal", "ic_0"]
    rhs = [P.random_rhs(A.n_rows, 3 + i) for i, A in enumerate(probs)]

    def run(items):
        B = serve.batch(ctx)
        for A, b, k in items:
            B.add(A, b, "cg", k, max_iter=3000, rtol=1e-8)
        B.solve(mixed=mixed)
        return [B.result(i) for i in range(len(items))]

    together = run(list(zip(probs, rhs, kinds)))
    with tuning(ctx, grid_sweep=0):
        chunked = run(list(zip(probs, rhs, kinds)))
    for g, c in zip(together, chunked):
        assert g.error_code == 0 and g.iterations == c.iterations and np.array_equal(g.x, c.x)
    # a batch of one Jacobi system runs the fused Jacobi path instead of
    # sweeps, so alone-equals-in-mix is checked on the IC(0) systems
    for i, it in enumerate(zip(probs, rhs, kinds)):
        if it[2] != "ic_0":
            continue
        alone = run([it])[0]
        assert alone.error_code == 0 and together[i].iterations == alone.iterations
        assert np.array_equal(together[i].x, alone.x)


def test_grid_expired_waits_report_timeout_and_recover(ctx):
    # at one poll the waits on other warps and CTAs expire: the apply
    # reports MTLG_ERR_TIMEOUT with the context usable, and the next applies
    # at the default limit are bitwise the oracle's again
    from mtl4_b200 import _lib, itl
    A = P.convdiff_3d(40)
    v = np.random.default_rng(5).standard_normal(A.n_rows).astype(np.float32)
    want = O.port_pc_apply(A, "ilu_0", v)
    Pc = itl.pc.ilu_0(dev(A, ctx), np.float32)
    assert Pc.sweep_plan(np.float32)["kernel"] == "grid"
    assert np.array_equal(itl.solve(Pc, vec(v, ctx, np.float32)).numpy(), want)
    with tuning(ctx, spin_limit=1):
        with pytest.raises(_lib.device_timeout):
            itl.solve(Pc, vec(v, ctx, np.float32))
    for _ in range(2):
        assert np.array_equal(itl.solve(Pc, vec(v, ctx, np.float32)).numpy(), want)


def test_grid_expired_waits_in_a_solve_recover(ctx):
    from mtl4_b200 import _lib, itl, mtl
    A = P.convdiff_3d(32)
    _, b = P.rhs_from_solution(A, 1)
    Ad = dev(A, ctx)

    def solve(Pc):
        x = mtl.dense_vector(A.n_rows, np.float64, ctx)
        it = itl.basic_iteration(vec(b, ctx), 500, 1e-8)
        itl.bicgstab(Ad, x, vec(b, ctx), Pc, it)
        return x.numpy(), it

    Pa = itl.pc.ilu_0(Ad, np.float64)
    Pb = itl.pc.ilu_0(Ad, np.float64)
    x0, it0 = solve(Pa)
    with tuning(ctx, spin_limit=1):
        with pytest.raises(_lib.device_timeout):
            solve(Pb)
    x1, it1 = solve(itl.pc.ilu_0(Ad, np.float64))
    x2, it2 = solve(Pa)
    assert it0.is_converged() and it1.iterations() == it0.iterations() and np.array_equal(x1, x0)
    assert it2.iterations() == it0.iterations() and np.array_equal(x2, x0)


@pytest.mark.parametrize("kind", ["ilu_0", "ic_0"])
def test_flat_sweep_after_grid_setup(ctx, kind):
    # a preconditioner set up with the grid layout only gets its flat layout
    # on first need (values copied from the grid layout): a flat-sweep apply
    # (sweep_kernel 1) and the factor download are the oracle's bit for bit
    from mtl4_b200 import itl
    A = P.vardiff_3d((40, 36, 9), sigma=0.7, seed=9, beta=(0.2, 0.1, 0.05))
    Ad = dev(A, ctx)
    x = np.random.default_rng(7).standard_normal(A.n_rows)
    for st in (np.float64, np.float32):
        Pc = getattr(itl.pc, kind)(Ad, st)
        assert Pc.sweep_plan(np.float64)["kernel"] == "grid"
        with tuning(ctx, sweep_kernel=1):
            y = itl.solve(Pc, vec(x, ctx)).numpy()
        assert np.array_equal(y, O.port_pc_apply(A, kind, x, storage_f32=(st == np.float32)))
        y2 = itl.solve(Pc, vec(x, ctx)).numpy()   # back on the grid sweep
        assert np.array_equal(y2, y)


@pytest.mark.parametrize("kind", ["ilu_0", "ic_0"])
def test_grid_factorization_equals_level_factorization(ctx, kind):
    # the pivots computed on the grid kernel (grid-stencil patterns) are the
    # level-scheduled factorization's bit for bit: the downloaded factors
    # match, for 2D and 3D grids, and for sides of 2 (ILU(0) keeps the
    # level-scheduled kernel there)
    from mtl4_b200 import itl
    for A in (P.vardiff_3d((17, 12, 5), sigma=1.0, seed=3, beta=(0.3, 0.2, 0.1)),
              P.vardiff_2d((45, 21), sigma=1.0, seed=4),
              P.vardiff_3d((9, 2, 6), sigma=0.5, seed=5)):
        Ad = dev(A, ctx)
        got = {}
        for grid in (1, 0):
            with tuning(ctx, grid_sweep=grid):
                Pc = getattr(itl.pc, kind)(Ad)
                got[grid] = [Pc.factor(w) for w in ("L", "U")]
        for (a, b) in zip(got[1], got[0]):
            for u, v in zip(a, b):
                assert np.array_equal(u, v)
