"""GPU parity of the chunked triangular sweeps (one CTA per chunk of
contiguous rows, level waves inside the chunk): preconditioner applies equal
the oracle bit for bit at chunk sizes that put most dependencies in other
chunks (32 rows), in the same chunk (whole matrix), and in between; waves
larger than a CTA are split; the chunked and the flat level-order kernels give
identical results; batched solves over many-chunk factors equal standalone
solves.  Grid-stencil matrices run here with the grid layout switched off
(grid_sweep 0), so the chunked kernel is the one under test."""
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


def random_banded_spd(n, band=40, per_row=3, seed=11):
    """Symmetric pattern with random off-diagonals within a band, strictly
    diagonally dominant: irregular levels and row lengths."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for i in range(n):
        lo = max(0, i - band)
        for j in (rng.choice(np.arange(lo, i), size=min(per_row, i - lo), replace=False) if i > 0 else []):
            v = -rng.uniform(0.1, 1.0)
            rows += [i, int(j)]
            cols += [int(j), i]
            vals += [v, v]
    rows = np.array(rows, np.int64)
    cols = np.array(cols, np.int64)
    vals = np.array(vals)
    diag = np.zeros(n)
    np.add.at(diag, rows, np.abs(vals))
    rows = np.concatenate([rows, np.arange(n)])
    cols = np.concatenate([cols, np.arange(n)])
    vals = np.concatenate([vals, diag + 1.0])
    return P._from_coo(n, rows, cols, vals)


def paired_blocks(n):
    """2x2 diagonal blocks: every other row is level 0, so a chunk's first
    wave holds half its rows (split across several CTA-sized waves)."""
    rows, cols, vals = [], [], []
    for i in range(0, n - 1, 2):
        rows += [i, i, i + 1, i + 1]
        cols += [i, i + 1, i, i + 1]
        vals += [4.0, -1.0, -1.0, 4.0]
    if n % 2:
        rows.append(n - 1); cols.append(n - 1); vals.append(4.0)
    return P._from_coo(n, np.array(rows), np.array(cols), np.array(vals))


PROBLEMS = {
    "vardiff2d_96": lambda: P.vardiff_2d(96, sigma=1.0, seed=7),
    "convdiff3d_20": lambda: P.convdiff_3d(20),
    "banded_6000": lambda: random_banded_spd(6000),
}


@pytest.mark.parametrize("name", list(PROBLEMS))
@pytest.mark.parametrize("chunk_rows", [32, 200, 4096, 32768])
def test_chunked_apply_matches_oracle(ctx, name, chunk_rows):
    from mtl4_b200 import itl
    A = PROBLEMS[name]()
    x = np.random.default_rng(5).standard_normal(A.n_rows)
    with tuning(ctx, grid_sweep=0, chunk_rows=chunk_rows, sweep_kernel=0):
        Ad = dev(A, ctx)
        for kind in ("ilu_0", "ic_0"):
            for mode in ("f64", "f64s32", "f32"):
                storage = np.float32 if mode != "f64" else np.float64
                vt = np.float32 if mode == "f32" else np.float64
                Pc = getattr(itl.pc, kind)(Ad, storage)
                y = itl.solve(Pc, vec(x.astype(vt), ctx, vt)).numpy()
                if mode == "f32":
                    ref = O.port_pc_apply(A, kind, x.astype(np.float32))
                else:
                    ref = O.port_pc_apply(A, kind, x, storage_f32=(mode == "f64s32"))
                assert np.array_equal(y, ref), (name, chunk_rows, kind, mode)


@pytest.mark.parametrize("cluster", [1, 2, 4, 8])
def test_cluster_pushes_match_oracle(ctx, cluster):
    # neighbouring chunks in one thread-block cluster hand their results over
    # through shared memory; runs of chunks cross cluster groups, and a group
    # may hold more chunks than fit at once
    from mtl4_b200 import itl
    A = P.vardiff_3d(24, sigma=1.0, seed=5, beta=(0.05, 0.02, 0.01))
    x = np.random.default_rng(12).standard_normal(A.n_rows)
    for chunk_rows in (96, 576, 2304):
        with tuning(ctx, grid_sweep=0, chunk_rows=chunk_rows, sweep_kernel=0, sweep_cluster=cluster):
            Ad = dev(A, ctx)
            for kind, dt in (("ilu_0", np.float64), ("ic_0", np.float32)):
                Pc = getattr(itl.pc, kind)(Ad, dt)
                assert Pc.sweep_plan(dt)["chunks"] > 1
                for _ in range(2):
                    y = itl.solve(Pc, vec(x.astype(dt), ctx, dt)).numpy()
                    assert np.array_equal(y, O.port_pc_apply(A, kind, x.astype(dt))), (chunk_rows, kind)


@pytest.mark.parametrize("cluster", [1, 8])
def test_batch_cluster_groups_match_standalone(ctx, cluster):
    # chunk runs of several systems packed into the groups of one cluster
    from mtl4_b200 import itl, mtl, serve
    probs = [P.vardiff_3d(m, sigma=0.5, seed=m, beta=(0.05, 0.02, 0.01)) for m in (7, 9, 12, 15)]
    rhs = [P.random_rhs(A.n_rows, 4) for A in probs]
    with tuning(ctx, grid_sweep=0, chunk_rows=256, sweep_kernel=0, sweep_cluster=cluster):
        B = serve.batch(ctx)
        for A, b in zip(probs, rhs):
            B.add(A, b, "bicgstab", "ilu_0", max_iter=2000, rtol=1e-8)
        B.solve(mixed=False)
        for i, (A, b) in enumerate(zip(probs, rhs)):
            Ad = mtl.compressed2D.from_problem(A, ctx)
            x = mtl.dense_vector(A.n_rows, np.float64, ctx)
            bd = mtl.dense_vector(b, np.float64, ctx)
            it = itl.basic_iteration(bd, 2000, 1e-8)
            itl.bicgstab(Ad, x, bd, itl.pc.ilu_0(Ad), it)
            r = B.result(i)
            assert r.error_code == 0
            assert r.iterations == it.iterations()
            assert np.array_equal(r.x, x.numpy())


def test_wave_split_beyond_cta(ctx):
    from mtl4_b200 import itl
    A = paired_blocks(9001)
    x = np.random.default_rng(3).standard_normal(A.n_rows)
    with tuning(ctx, grid_sweep=0, chunk_rows=8192, sweep_kernel=0):
        Pc = itl.pc.ilu_0(dev(A, ctx))
        y = itl.solve(Pc, vec(x, ctx)).numpy()
    assert np.array_equal(y, O.port_pc_apply(A, "ilu_0", x))


def test_chunked_equals_flat(ctx):
    from mtl4_b200 import itl
    A = P.vardiff_3d(24, sigma=1.0, seed=3, beta=(0.05, 0.02, 0.01))
    x = np.random.default_rng(9).standard_normal(A.n_rows)
    with tuning(ctx, grid_sweep=0, chunk_rows=1024, sweep_kernel=0):
        Ad = dev(A, ctx)
        pcs = [itl.pc.ilu_0(Ad), itl.pc.ic_0(Ad, np.float32)]
    for Pc in pcs:
        with tuning(ctx, grid_sweep=0, sweep_kernel=0):
            y0 = itl.solve(Pc, vec(x, ctx)).numpy()
        with tuning(ctx, grid_sweep=0, sweep_kernel=1):
            y1 = itl.solve(Pc, vec(x, ctx)).numpy()
        assert np.array_equal(y0, y1)


@pytest.mark.parametrize("solver,kind", [("cg", "ic_0"), ("bicgstab", "ilu_0")])
def test_flat_solve_after_chunked_setup(ctx, solver, kind):
    # a preconditioner set up with the chunked layout only gets its flat
    # entries on first need: here a solve under sweep_kernel 1 (flat level
    # order), which must give the chunked solve's iterations and x exactly
    from mtl4_b200 import itl, mtl
    A = P.vardiff_3d(20, sigma=1.0, seed=5, beta=(0.05, 0.02, 0.01))
    b = np.random.default_rng(3).standard_normal(A.n_rows)
    out = []
    for flat in (0, 1):
        with tuning(ctx, grid_sweep=0, chunk_rows=1024, sweep_kernel=0):
            Ad = dev(A, ctx)
            Pc = getattr(itl.pc, kind)(Ad)
        with tuning(ctx, grid_sweep=0, sweep_kernel=flat):
            x = mtl.dense_vector(A.n_rows, np.float64, ctx)
            bd = vec(b, ctx)
            it = itl.basic_iteration(bd, 1000, 1e-10)
            getattr(itl, solver)(Ad, x, bd, Pc, it)
            out.append((it.iterations(), x.numpy()))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])


def test_chunked_repeated_applies_keep_invariants(ctx):
    # the sweeps reset their buffers to the sentinel row by row; a second and
    # third apply on the same preconditioner must give the same result
    from mtl4_b200 import itl
    A = P.vardiff_2d(64, sigma=1.0, seed=2)
    x = np.random.default_rng(4).standard_normal(A.n_rows)
    with tuning(ctx, grid_sweep=0, chunk_rows=256, sweep_kernel=0):
        Pc = itl.pc.ic_0(dev(A, ctx))
        ys = [itl.solve(Pc, vec(x, ctx)).numpy() for _ in range(3)]
    assert all(np.array_equal(ys[0], y) for y in ys[1:])
    assert np.array_equal(ys[0], O.port_pc_apply(A, "ic_0", x))


@pytest.mark.parametrize("solver,kind", [("cg", "ic_0"), ("bicgstab", "ilu_0")])
def test_batch_many_chunks_matches_standalone(ctx, solver, kind):
    from mtl4_b200 import itl, mtl, serve
    probs = [P.vardiff_3d(m, sigma=0.5, seed=m, beta=(0.05, 0.02, 0.01)) for m in (10, 14, 17)]
    rhs = [P.random_rhs(A.n_rows, 3) for A in probs]
    with tuning(ctx, grid_sweep=0, chunk_rows=128, sweep_kernel=0):
        B = serve.batch(ctx)
        for A, b in zip(probs, rhs):
            B.add(A, b, solver, kind, max_iter=2000, rtol=1e-8)
        B.solve(mixed=False)
        for i, (A, b) in enumerate(zip(probs, rhs)):
            Ad = mtl.compressed2D.from_problem(A, ctx)
            x = mtl.dense_vector(A.n_rows, np.float64, ctx)
            bd = mtl.dense_vector(b, np.float64, ctx)
            it = itl.basic_iteration(bd, 2000, 1e-8)
            getattr(itl, solver)(Ad, x, bd, getattr(itl.pc, kind)(Ad), it)
            r = B.result(i)
            assert r.error_code == 0
            assert r.iterations == it.iterations()
            assert np.array_equal(r.x, x.numpy())


@pytest.mark.parametrize("cluster", [1, 4])
def test_expired_dependency_waits_report_timeout_and_recover(ctx, cluster):
    # the context's spin_limit bounds every dependency wait of the sweeps; at
    # one poll the chunks' waits on earlier chunks expire: the apply reports
    # MTLG_ERR_TIMEOUT (device_timeout) with the context still usable, and
    # the next apply at the default limit is bitwise the oracle's again.  The
    # chunks' own staging copies keep their fixed bound, so nothing is in
    # flight when a CTA ends.
    from mtl4_b200 import _lib, itl
    A = P.convdiff_3d(40)
    v = np.random.default_rng(5).standard_normal(A.n_rows).astype(np.float32)
    want = O.port_pc_apply(A, "ilu_0", v)
    with tuning(ctx, grid_sweep=0, chunk_rows=1600, sweep_cluster=cluster):
        Pc = itl.pc.ilu_0(dev(A, ctx), np.float32)
        assert Pc.sweep_plan(np.float32)["chunks"] >= 16
        assert np.array_equal(itl.solve(Pc, vec(v, ctx, np.float32)).numpy(), want)
        with tuning(ctx, grid_sweep=0, spin_limit=1):
            with pytest.raises(_lib.device_timeout):
                itl.solve(Pc, vec(v, ctx, np.float32))
        for _ in range(2):
            assert np.array_equal(itl.solve(Pc, vec(v, ctx, np.float32)).numpy(), want)


def test_expired_waits_in_a_solve_report_timeout_and_recover(ctx):
    # a solve whose loop graphs were built at a one-poll limit: the sweeps'
    # waits expire inside the graph, the solve reports MTLG_ERR_TIMEOUT, and
    # the preconditioner's sweep state is re-armed; later solves (sets built
    # at the default limit) are bitwise the earlier ones
    from mtl4_b200 import _lib, itl, mtl
    A = P.convdiff_3d(32)
    _, b = P.rhs_from_solution(A, 1)
    Ad = dev(A, ctx)

    def solve(Pc):
        x = mtl.dense_vector(A.n_rows, np.float64, ctx)
        it = itl.basic_iteration(vec(b, ctx), 500, 1e-8)
        itl.bicgstab(Ad, x, vec(b, ctx), Pc, it)
        return x.numpy(), it

    with tuning(ctx, grid_sweep=0, chunk_rows=1024):
        Pa = itl.pc.ilu_0(Ad, np.float64)
        Pb = itl.pc.ilu_0(Ad, np.float64)
        x0, it0 = solve(Pa)
        with tuning(ctx, grid_sweep=0, spin_limit=1):
            with pytest.raises(_lib.device_timeout):
                solve(Pb)
        Pc = itl.pc.ilu_0(Ad, np.float64)
        x1, it1 = solve(Pc)
        x2, it2 = solve(Pa)
    assert it0.is_converged() and it1.iterations() == it0.iterations() and np.array_equal(x1, x0)
    assert it2.iterations() == it0.iterations() and np.array_equal(x2, x0)
