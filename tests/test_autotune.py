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
