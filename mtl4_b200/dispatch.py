"""Several GPUs, one process each: batches and request streams shard by whole
systems, with no collective on the data path (no reference counterpart: MTL4
has no multi-process code).

Every rank computes the same size-balanced assignment
(``mtlg_partition_systems``: longest processing time first, cost = nnz + n),
solves its share on its own GPU with the single-GPU engine, and the results
are gathered on the host of rank 0 (``torch.distributed.gather_object``, the
process group's host transport) and put back in submission order.

``solve_sharded`` takes the per-rank solve as a callable, so the same
partition-and-gather path runs with the GPU batch engine in production and
with any host solver where no GPU is present.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Sequence

import numpy as np

from . import _lib


def system_cost(A) -> int:
    """Work estimate of one solve per iteration: entries plus rows."""
    return int(A.nnz) + int(A.n_rows)


def partition(costs: Sequence[int], n_parts: int) -> tuple[np.ndarray, np.ndarray]:
    """part_of[i] for every system and the total cost of each part (host
    only, deterministic)."""
    c = np.ascontiguousarray(np.asarray(costs, dtype=np.int64))
    part_of = np.zeros(c.size, dtype=np.int32)
    load = np.zeros(int(n_parts), dtype=np.int64)
    st = _lib.lib().mtlg_partition_systems(c.size, C.c_void_p(c.ctypes.data), int(n_parts),
                                                   C.c_void_p(part_of.ctypes.data), C.c_void_p(load.ctypes.data))
    _lib.check(st, "partition_systems")
    return part_of, load


def shard(n_items: int, part_of: np.ndarray, rank: int) -> list[int]:
    """Indices (in submission order) that `rank` solves."""
    return [i for i in range(n_items) if int(part_of[i]) == rank]


def gather(local: dict, rank: int, world: int) -> dict | None:
    """Merge every rank's {index: result} on rank 0 (None elsewhere)."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist
    parts = [None] * world if rank == 0 else None
    dist.gather_object(local, parts, dst=0)
    if rank != 0:
        return None
    merged = {}
    for p in parts:
        merged.update(p)
    return merged


def solve_sharded(systems: Sequence, rhs: Sequence[np.ndarray], solve_share: Callable[[list[int]], dict],
                  rank: int = 0, world: int = 1) -> list | None:
    """Partition `systems` over `world` ranks, run `solve_share(indices)` (a
    dict index -> result for this rank's systems) and gather.  Rank 0 gets
    the results in submission order, the other ranks None."""
    part_of, _ = partition([system_cost(A) for A in systems], world)
    mine = shard(len(systems), part_of, rank)
    local = solve_share(mine)
    if set(local) != set(mine):
        raise RuntimeError(f"rank {rank} returned results for {sorted(set(local) ^ set(mine))[:8]} ...")
    merged = gather(local, rank, world)
    if merged is None:
        return None
    return [merged[i] for i in range(len(systems))]


def gpu_batch_share(systems, rhs, specs, ctx, mixed: bool, rtol: float = 1e-8, inner_rtol: float = 1e-5,
                    max_iter: int = 3000):
    """The per-rank solve for `solve_sharded` on a GPU: this rank's systems as
    one batch on its device (every system keeps its own iteration state, so
    its result is the one it has alone)."""
    from . import serve

    def run(indices: list[int]) -> dict:
        if not indices:
            return {}
        B = serve.batch(ctx)
        for i in indices:
            B.add(systems[i], rhs[i], specs[i].solver, specs[i].pc, max_iter=max_iter, rtol=rtol)
        B.solve(mixed=mixed, rtol=rtol, inner_rtol=inner_rtol)
        return {i: B.result(k) for k, i in enumerate(indices)}

    return run


def assign_stream(costs: Sequence[int], n_parts: int) -> np.ndarray:
    """Online assignment of a request stream in arrival order: each request
    goes to the rank with the least cost assigned so far (ties: lowest
    rank), so a rank can take its requests as they arrive."""
    load = np.zeros(int(n_parts), dtype=np.int64)
    out = np.zeros(len(costs), dtype=np.int32)
    for i, c in enumerate(costs):
        r = int(np.argmin(load))
        out[i] = r
        load[r] += int(c)
    return out
