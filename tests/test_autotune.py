"""Autotuner host logic (no GPU): cache keys, persistence, selection."""
import numpy as np
import pytest

from mtl4_b200 import autotune, problems as P


def test_row_histogram_buckets():
    rp = np.array([0, 0, 1, 3, 7, 15, 16])      # lengths 0,1,2,4,8,1
    h = autotune.row_histogram(rp)
    assert h[:5] == [1, 2, 1, 1, 1]


def test_signature_groups_same_shape_and_separates_others():
    a = autotune.signature("B200", "sweep", "float32", P.laplacian_2d(32))
    b = autotune.signature("B200", "sweep", "float32", P.laplacian_2d(32))
    c = autotune.signature("B200", "sweep", "float32", P.laplacian_2d(33))
    d = autotune.signature("B200", "sweep", "float64", P.laplacian_2d(32))
    assert a == b and a != c and a != d


def test_best_of_picks_fastest_and_reports_all():
    cands = [{"k": 1}, {"k": 2}, {"k": 3}]
    best, t = autotune.best_of(cands, lambda c: {1: 3.0, 2: 1.0, 3: 2.0}[c["k"]])
    assert best == {"k": 2} and len(t) == 3


def test_cache_persists(tmp_path):
    path = tmp_path / "tune.json"
    c = autotune.Cache(path)
    c.put("key", {"choice": {"sweep_blocks": 148}})
    c2 = autotune.Cache(path)
    assert c2.get("key")["choice"]["sweep_blocks"] == 148
    assert c2.get("missing") is None


def test_sweep_candidates_cover_grid_and_backoff():
    cs = autotune.sweep_candidates(148)
    assert {c["sweep_blocks"] for c in cs} == {74, 148, 222, 296}
    assert {c["sweep_sleep_ns"] for c in cs} == {0, 64}


def test_coordinate_search_keeps_best_per_knob_and_measures_once():
    # separable cost: best is a=2, b=30; each distinct setting measured once
    calls = []

    def measure(c):
        calls.append((c["a"], c["b"]))
        return {1: 3.0, 2: 1.0, 3: 2.0}[c["a"]] + {10: 5.0, 20: 4.0, 30: 0.5}[c["b"]]

    best, t = autotune.coordinate_search({"a": (1, 2, 3), "b": (10, 20, 30)}, {"a": 1, "b": 10}, measure)
    assert best == {"a": 2, "b": 30}
    assert len(calls) == len(set(calls)) == len(t)
    assert (1, 10) in calls and (2, 30) in calls


def test_batch_signature_tracks_set_shape():
    s1 = [P.laplacian_2d(16), P.laplacian_2d(20)]
    s2 = [P.laplacian_2d(16), P.laplacian_2d(20)]
    s3 = [P.laplacian_2d(16)]
    a = autotune.batch_signature("B200", "batch:cg:ic_0:fp64", "float64", s1)
    assert a == autotune.batch_signature("B200", "batch:cg:ic_0:fp64", "float64", s2)
    assert a != autotune.batch_signature("B200", "batch:cg:ic_0:fp64", "float64", s3)
    assert a != autotune.batch_signature("B200", "batch:cg:ic_0:mixed", "float64", s1)


def test_cached_choice_is_applied_without_measuring(tmp_path):
    # a cache hit sets the knobs on the context and measures nothing
    class FakeCtx:
        def __init__(self):
            self.knobs = {}

        def set_tuning(self, k, v):
            self.knobs[k] = v

    A = P.laplacian_2d(24)

    class Dev:
        shape = (A.n_rows, A.n_cols)
        nnz = A.nnz
        host_row_ptr = A.row_ptr

    cache = autotune.Cache(tmp_path / "c.json")
    key = autotune.signature("G", "pc:ic_0", "float32", autotune._Shape(A.n_rows, A.nnz, A.row_ptr))
    cache.put(key, {"choice": {"chunk_rows": 4096, "sweep_cluster": 2}})
    ctx = FakeCtx()
    choice, hit = autotune.tune_pc(ctx, Dev(), "ic_0", np.float32, cache=cache, gpu="G")
    assert hit and ctx.knobs == {"chunk_rows": 4096, "sweep_cluster": 2}


@pytest.mark.gpu
def test_autotune_wired_into_pc_solve_mult_and_batch(tmp_path):
    from mtl4_b200 import itl, mtl, serve
    from oracle import oracle as O
    ctx = mtl.context(0)
    cache = autotune.Cache(tmp_path / "w.json")
    ctx.enable_autotune(cache)
    try:
        A = P.vardiff_2d(96, seed=3)
        Ad = mtl.compressed2D.from_problem(A, ctx)
        Pc = itl.pc.ic_0(Ad, np.float32)          # tunes grid_warps (a grid stencil), else chunk_rows / sweep_cluster
        assert ("pc", "ic_0", "float32") in Ad._tuned
        ch = Ad._tuned[("pc", "ic_0", "float32")]
        if "grid_warps" in ch:
            assert ch["grid_warps"] in autotune.GRID_WARPS and Pc.sweep_plan(np.float32)["kernel"] == "grid"
        else:
            assert ch["chunk_rows"] in autotune.CHUNK_ROWS and ch["sweep_cluster"] in autotune.SWEEP_CLUSTERS
        # the tuned preconditioner is still the reference's apply
        r = np.random.default_rng(1).standard_normal(A.n_rows).astype(np.float32)
        assert np.array_equal(itl.solve(Pc, mtl.dense_vector(r, np.float32, ctx)).numpy(),
                              O.port_pc_apply(A, "ic_0", r))
        b = np.ones(A.n_rows)
        x = mtl.dense_vector(A.n_rows, np.float64, ctx)
        bd = mtl.dense_vector(b, np.float64, ctx)
        Pd = itl.pc.ic_0(Ad, np.float64)
        it = itl.basic_iteration(bd, 2000, 1e-8)
        itl.cg(Ad, x, bd, Pd, it)                  # tunes vec_ctas_per_sm
        assert "vec" in Ad._tuned and it.is_converged()
        assert np.linalg.norm(A.matvec(x.numpy()) - b) <= 1.05e-8 * np.linalg.norm(b)
        y = mtl.dense_vector(A.n_rows, np.float64, ctx)
        mtl.mult(Ad, bd, y)                        # tunes spmv_kernel
        assert Ad._tuned["spmv"]["spmv_kernel"] in autotune.SPMV_KERNELS
        assert np.array_equal(y.numpy(), O.port_spmv(A, b))
        n_keys = len(cache.data)
        assert n_keys >= 3
        # a second matrix of the same class is served from the cache
        Ad2 = mtl.compressed2D.from_problem(A, ctx)
        itl.pc.ic_0(Ad2, np.float32)
        assert Ad2._tuned[("pc", "ic_0", "float32")] == ch and len(cache.data) == n_keys
        # batched passes
        bt = serve.batch(ctx)
        systems = [P.laplacian_2d(40 + 4 * i) for i in range(6)]
        for S in systems:
            bt.add(S, np.ones(S.n_rows), "cg", "ic_0")
        bt.solve(mixed=True, tune=cache)
        for i, S in enumerate(systems):
            r = bt.result(i)
            assert r.error_code == 0
            assert np.linalg.norm(S.matvec(r.x) - 1.0) <= 1.05e-8 * np.sqrt(S.n_rows)
        assert len(cache.data) == n_keys + 1
    finally:
        ctx.disable_autotune()
        for k, v in (("chunk_rows", 0), ("sweep_cluster", 0), ("vec_ctas_per_sm", 2), ("spmv_kernel", 0)):
            ctx.set_tuning(k, v)


@pytest.mark.gpu
def test_tune_sweeps_on_device(tmp_path):
    from mtl4_b200 import itl, mtl
    ctx = mtl.context(0)
    A = P.vardiff_2d(128, seed=1)
    Ad = mtl.compressed2D.from_problem(A, ctx)
    Pc = itl.pc.ic_0(Ad, np.float32)
    cache = autotune.Cache(tmp_path / "t.json")
    choice, hit = autotune.tune_sweeps(ctx, A, Pc, cache=cache, reps=1)
    assert not hit and ctx.get_tuning("sweep_blocks") == choice["sweep_blocks"]
    choice2, hit2 = autotune.tune_sweeps(ctx, A, Pc, cache=cache, reps=1)
    assert hit2 and choice2 == choice
    # still correct after tuning
    x = np.random.default_rng(0).standard_normal(A.n_rows).astype(np.float32)
    from oracle import oracle as O
    y = itl.solve(Pc, mtl.dense_vector(x, np.float32, ctx))
    assert np.array_equal(y.numpy(), O.port_pc_apply(A, "ic_0", x))
