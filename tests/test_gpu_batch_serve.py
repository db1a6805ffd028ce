"""GPU tests of batched and served solves: each system's result meets its
tolerance, batched results equal standalone solves, and a served request's
result is the same alone and in a mix of concurrent requests."""
import numpy as np
import pytest

from mtl4_b200 import problems as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def small_specs(count=12, seed=4):
    specs = P.batch_specs(count, n_lo=500, n_hi=20_000, seed=seed)
    out = []
    for sp in specs:
        A = sp.build()
        b = P.random_rhs(A.n_rows, sp.seed)
        out.append((sp, A, b))
    return out


def relres(A, x, b):
    return np.linalg.norm(A.matvec(x) - b) / np.linalg.norm(b)


@pytest.mark.parametrize("mixed", [False, True])
def test_batch_uneven_systems(ctx, mixed):
    from mtl4_b200 import serve
    sys_ = small_specs()
    B = serve.batch(ctx)
    for sp, A, b in sys_:
        B.add(A, b, "cg", sp.pc, max_iter=3000, rtol=1e-8)
    B.solve(mixed=mixed, rtol=1e-8, inner_rtol=1e-4)
    for i, (sp, A, b) in enumerate(sys_):
        r = B.result(i)
        assert r.error_code == 0, (i, r)
        assert relres(A, r.x, b) <= 1.05e-8
        if not mixed:
            ref = O.port_solve(A, b, "cg", sp.pc, max_iter=3000, rtol=1e-8)
            assert abs(r.iterations - ref["iterations"]) <= 2


def test_batch_matches_standalone_bitwise(ctx):
    # IC(0) systems take the same kernels and the same per-system reduction
    # order in a batch as alone
    from mtl4_b200 import itl, mtl, serve
    sys_ = [s for s in small_specs(10, seed=9) if s[0].pc == "ic_0"][:4]
    B = serve.batch(ctx)
    for sp, A, b in sys_:
        B.add(A, b, "cg", "ic_0", max_iter=3000, rtol=1e-8)
    B.solve(mixed=False)
    for i, (sp, A, b) in enumerate(sys_):
        Ad = mtl.compressed2D.from_problem(A, ctx)
        x = mtl.dense_vector(A.n_rows, np.float64, ctx)
        bd = mtl.dense_vector(b, np.float64, ctx)
        it = itl.basic_iteration(bd, 3000, 1e-8)
        itl.cg(Ad, x, bd, itl.pc.ic_0(Ad), it)
        r = B.result(i)
        assert r.iterations == it.iterations()
        assert np.array_equal(r.x, x.numpy())


def test_batch_bicgstab_ilu0(ctx):
    from mtl4_b200 import serve
    B = serve.batch(ctx)
    probs = [P.vardiff_3d(m, sigma=0.5, seed=m, beta=(0.05, 0.02, 0.01)) for m in (8, 12, 16)]
    rhs = [P.random_rhs(A.n_rows, 7) for A in probs]
    for A, b in zip(probs, rhs):
        B.add(A, b, "bicgstab", "ilu_0", max_iter=1000, rtol=1e-8)
    B.solve(mixed=True)
    for i, (A, b) in enumerate(zip(probs, rhs)):
        r = B.result(i)
        assert r.error_code == 0 and relres(A, r.x, b) <= 1.05e-8


@pytest.mark.parametrize("mixed", [True, False])
def test_served_alone_equals_in_mix(ctx, mixed):
    served_alone_equals_in_mix(ctx, mixed)


def test_served_mix_in_clusters(ctx):
    # small chunks and 4-CTA clusters: every request spans several chunks,
    # cluster groups hold CTAs without a chunk, and slots (slot 0 among
    # them) fall free while the others still run
    old = {k: ctx.get_tuning(k) for k in ("chunk_rows", "sweep_cluster", "grid_sweep")}
    try:
        ctx.set_tuning("chunk_rows", 512)
        ctx.set_tuning("sweep_cluster", 4)
        ctx.set_tuning("grid_sweep", 0)   # the chunked kernel, also for grid-stencil requests
        served_alone_equals_in_mix(ctx, True)
    finally:
        for k, v in old.items():
            ctx.set_tuning(k, v)


def served_alone_equals_in_mix(ctx, mixed):
    from mtl4_b200 import serve
    sys_ = small_specs(10, seed=21)
    reqs = [(A, b, "cg", sp.pc, 3000) for sp, A, b in sys_]
    # an extra BiCGSTAB + ILU(0) request with convection
    Ac = P.vardiff_2d(40, sigma=1.0, seed=3, beta=(0.01, 0.02))
    reqs.append((Ac, P.random_rhs(Ac.n_rows, 1), "bicgstab", "ilu_0", 3000))
    alone = []
    for req in reqs:
        srv = serve.server(ctx, max_active=4, iters_per_step=8, mixed=mixed)
        res = serve.run_open_loop(srv, [req], [0.0])
        alone.append(res["results"][0])
        del srv
    srv = serve.server(ctx, max_active=4, iters_per_step=8, mixed=mixed)
    arrivals = np.linspace(0.0, 0.05, len(reqs))
    mix = serve.run_open_loop(srv, reqs, arrivals)
    assert mix["completed"] == len(reqs)
    for i, (A, b, *_rest) in enumerate(reqs):
        r_mix, r_alone = mix["results"][i], alone[i]
        assert r_mix.error_code == 0
        assert relres(A, r_mix.x, b) <= 1.05e-8
        assert r_mix.iterations == r_alone.iterations
        assert np.array_equal(r_mix.x, r_alone.x)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["active"] == 0


def test_server_admission_and_cancel(ctx):
    from mtl4_b200 import _lib, serve
    A = P.vardiff_2d(64, sigma=1.0, seed=1)
    b = P.random_rhs(A.n_rows, 2)
    srv = serve.server(ctx, hbm_budget=200_000, max_active=2)
    with pytest.raises(_lib.MtlError):
        srv.submit(A, b, "cg", "ic_0")            # can never fit the budget
    assert srv.stats()["rejected"] == 1
    srv2 = serve.server(ctx, max_active=2, iters_per_step=4)
    ids = [srv2.submit(A, b, "cg", "ic_0") for _ in range(3)]
    srv2.step()                                   # two admitted, one queued
    st = srv2.stats()
    assert st["active"] == 2 and st["queued"] == 1
    srv2.cancel(ids[0])
    for _ in range(2000):
        srv2.step()
        if all(srv2.poll(i) is not None for i in ids[1:] if i in srv2.n):
            break
    assert srv2.stats()["cancelled"] == 1


def test_server_admits_by_free_device_memory(ctx):
    # no byte budget: admission by the device's free memory less a reserve.
    # The free figure is simulated (context tuning) so that one request fits
    # at a time; the others wait in the queue and are admitted as earlier
    # ones retire; a request larger than free + held memory is refused.
    from mtl4_b200 import _lib, serve
    A = P.vardiff_2d(48, sigma=1.0, seed=4)
    b = P.random_rhs(A.n_rows, 3)
    probe = serve.server(ctx, max_active=4, iters_per_step=8)
    probe.submit(A, b, "cg", "ic_0")
    probe.step()
    one = probe.stats()["bytes_in_use"]
    assert one > 0
    del probe
    old = {k: ctx.get_tuning(k) for k in ("admission_free_bytes", "admission_reserve_bytes")}
    ctx.set_tuning("admission_free_bytes", int(one * 1.5))
    ctx.set_tuning("admission_reserve_bytes", 0)
    try:
        srv = serve.server(ctx, max_active=4, iters_per_step=8)
        ids = [srv.submit(A, b, "cg", "ic_0") for _ in range(3)]
        most = 0
        done = {}
        for _ in range(5000):
            srv.step()
            most = max(most, srv.stats()["active"])
            for i in ids:
                if i not in done and i in srv.n:
                    r = srv.poll(i)
                    if r is not None:
                        done[i] = r
            if len(done) == len(ids):
                break
        assert most == 1 and len(done) == 3
        assert all(r.error_code == 0 and relres(A, r.x, b) <= 1.05e-8 for r in done.values())
        big = P.vardiff_2d(160, sigma=1.0, seed=4)
        with pytest.raises(_lib.MtlError):
            srv.submit(big, P.random_rhs(big.n_rows, 3), "cg", "ic_0")   # more than free + held
    finally:
        for k, v in old.items():
            ctx.set_tuning(k, v)


def test_batch_and_server_finish_stalled_refinement_in_fp64(ctx):
    # the served stream's request 33 is too ill-conditioned for the FP32 inner
    # solve; batch and server finish it in FP64 and report that they did
    from mtl4_b200 import serve
    sp = P.request_specs(20000)[33]
    A = sp.build()
    b = P.random_rhs(A.n_rows, sp.seed)
    B = serve.batch(ctx)
    B.add(A, b, "bicgstab", "ilu_0", max_iter=2000, rtol=1e-8)
    B.solve(mixed=True, rtol=1e-8, inner_rtol=1e-4)
    r = B.result(0)
    assert r.error_code == 0 and r.fp64_fallback and relres(A, r.x, b) <= 1.05e-8
    srv = serve.server(ctx, max_active=4, iters_per_step=16, mixed=True, rtol=1e-8, inner_rtol=1e-4)
    out = serve.run_open_loop(srv, [(A, b, "bicgstab", "ilu_0", 2000)], np.zeros(1), timeout_s=120.0)
    r = out["results"][0]
    assert r is not None and r.error_code == 0 and r.fp64_fallback and relres(A, r.x, b) <= 1.05e-8
