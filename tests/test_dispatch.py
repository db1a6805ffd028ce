"""Several GPUs by whole systems (no GPU needed): the size-balanced partition
and the shard / gather path, run as two gloo ranks on the CPU with the
oracle's solver standing in for each rank's GPU batch.  The gathered results
must equal the single-rank run exactly, in submission order."""
import os
import socket

import numpy as np
import pytest

from mtl4_b200 import dispatch
from mtl4_b200 import problems as P


def test_partition_is_size_balanced_and_deterministic():
    costs = [100, 7, 50, 50, 3, 90, 10, 10]
    part, load = dispatch.partition(costs, 3)
    # LPT: 100 -> p0, 90 -> p1, 50 -> p2, 50 -> p2 (100), 10 -> p1 (100), 10 -> p0 (110), 7 -> p1, 3 -> p2
    assert part.tolist() == [0, 1, 2, 2, 2, 1, 1, 0]
    assert load.tolist() == [110, 107, 103]
    assert load.sum() == sum(costs)
    again, _ = dispatch.partition(costs, 3)
    assert np.array_equal(part, again)
    one, l1 = dispatch.partition(costs, 1)
    assert np.all(one == 0) and l1.tolist() == [sum(costs)]
    empty, l0 = dispatch.partition([], 4)
    assert empty.size == 0 and l0.tolist() == [0, 0, 0, 0]


def test_partition_balances_the_uneven_batch():
    specs = P.batch_specs(1024)
    costs = [sp.n * (5 if sp.dims == 2 else 7) + sp.n for sp in specs]
    for world in (2, 4, 8):
        _, load = dispatch.partition(costs, world)
        assert load.max() <= 1.02 * load.mean(), (world, load)


def test_partition_rejects_bad_arguments():
    from mtl4_b200 import _lib
    with pytest.raises(_lib.MtlError):
        dispatch.partition([1, -2], 2)
    with pytest.raises(_lib.MtlError):
        dispatch.partition([1, 2], 0)


def test_stream_assignment_is_online_greedy():
    assert dispatch.assign_stream([5, 1, 1, 1, 5], 2).tolist() == [0, 1, 1, 1, 1]


def _systems():
    specs = P.batch_specs(12, n_lo=200, n_hi=3000, seed=4)
    systems = [sp.build() for sp in specs]
    rhs = [P.random_rhs(A.n_rows, sp.seed) for sp, A in zip(specs, systems)]
    return specs, systems, rhs


def _oracle_share(specs, systems, rhs):
    from oracle import oracle as O

    def run(indices):
        return {i: O.port_solve(systems[i], rhs[i], specs[i].solver, specs[i].pc, max_iter=3000, rtol=1e-8)["x"]
                for i in indices}
    return run


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs, systems, rhs = _systems()
        res = dispatch.solve_sharded(systems, rhs, _oracle_share(specs, systems, rhs), rank, world)
        part, _ = dispatch.partition([dispatch.system_cost(A) for A in systems], world)
        np.save(os.path.join(out_dir, f"part{rank}.npy"), part)
        if rank == 0:
            np.savez(os.path.join(out_dir, "gathered.npz"), *res)
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_gather_the_single_rank_results(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    specs, systems, rhs = _systems()
    single = dispatch.solve_sharded(systems, rhs, _oracle_share(specs, systems, rhs), 0, 1)
    got = np.load(tmp_path / "gathered.npz")
    assert len(got.files) == len(systems)
    for i in range(len(systems)):
        assert np.array_equal(got[f"arr_{i}"], single[i]), i
    p0, p1 = np.load(tmp_path / "part0.npy"), np.load(tmp_path / "part1.npy")
    assert np.array_equal(p0, p1) and set(p0.tolist()) == {0, 1}
