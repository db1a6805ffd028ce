"""Batched and served solves on one GPU (no reference counterpart).

``batch``   -- many independent systems solved together by the same kernels.
``server``  -- continuous batching: requests arrive while others are on the
               device and are admitted as slots and device memory free up.
``run_open_loop`` drives a server with an open-loop Poisson arrival stream
and reports throughput with p50/p99 latency.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check
from .mtl import context, default_context

_SOLVER = {"cg": _lib.CG, "bicgstab": _lib.BICGSTAB}
_PC = {"identity": _lib.PC_IDENTITY, "diagonal": _lib.PC_DIAGONAL, "ilu_0": _lib.PC_ILU0, "ic_0": _lib.PC_IC0}


def _p(a):
    return C.c_void_p(a.ctypes.data)


@dataclass
class Result:
    x: np.ndarray
    iterations: int
    error_code: int
    status: int
    outer: int
    resid: float
    relresid: float
    seconds: float = 0.0
    fp64_fallback: bool = False   # mixed precision finished by a plain FP64 solve


def _result(x, r: _lib.IterResult) -> Result:
    return Result(x, r.iterations, r.error_code, r.status, r.outer_iterations, r.resid, r.relresid, r.seconds,
                  bool(r.fp64_fallback))


class batch:
    def __init__(self, ctx: context | None = None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        check(self.ctx._L.mtlg_batch_create(self.ctx.h, C.byref(h)), "batch_create")
        self.h = h
        self.sizes = []
        self.systems = []   # (A, solver, pc) of each system, for tune=True

    def add(self, A, b, solver="cg", pc="ic_0", max_iter=2000, rtol=1e-8, atol=0.0) -> int:
        rp = np.ascontiguousarray(A.row_ptr, np.int64)
        ci = np.ascontiguousarray(A.col, np.int32)
        v = np.ascontiguousarray(A.val, np.float64)
        bb = np.ascontiguousarray(b, np.float64)
        prm = _lib.IterParams(int(max_iter), 0, float(rtol), float(atol), -1.0)
        idx = C.c_int()
        check(self.ctx._L.mtlg_batch_add(self.h, A.n_rows, A.nnz, _p(rp), _p(ci), _p(v), _p(bb), _SOLVER[solver],
                                         _PC[pc], C.byref(prm), C.byref(idx)), "batch_add")
        self.sizes.append(A.n_rows)
        self.systems.append((A, solver, pc))
        return idx.value

    def solve(self, mixed: bool = False, rtol: float = 1e-8, inner_rtol: float = 1e-4, max_outer: int = 20,
              max_inner: int = 2000, tune=False):
        """Solves every system.  tune: True (or an autotune.Cache) first sets
        the context's batched-pass knobs for this set of systems (measured on
        a sample of them once per class, then cached)."""
        if tune:
            self.tune(mixed, cache=None if tune is True else tune)
        rp = _lib.RefineParams(int(max_outer), int(max_inner), 0, 0, float(rtol), float(inner_rtol))
        check(self.ctx._L.mtlg_batch_solve(self.h, _lib.F32 if mixed else _lib.F64, C.byref(rp)), "batch_solve")

    def tune(self, mixed: bool = False, cache=None):
        from . import autotune
        if not self.systems:
            return None
        kinds = {}
        for _, so, pc in self.systems:
            kinds[(so, pc)] = kinds.get((so, pc), 0) + 1
        solver, pc = max(kinds, key=kinds.get)
        cache = cache or self.ctx.autotune or autotune.Cache()
        return autotune.tune_batch(self.ctx, [A for A, _, _ in self.systems], solver, pc, mixed, cache=cache)[0]

    def result(self, i: int) -> Result:
        x = np.empty(self.sizes[i])
        r = _lib.IterResult()
        check(self.ctx._L.mtlg_batch_result(self.h, i, _p(x), C.byref(r)), "batch_result")
        return _result(x, r)

    def __len__(self):
        return len(self.sizes)

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                self.ctx._L.mtlg_batch_destroy(self.h)
        except Exception:
            pass


class server:
    def __init__(self, ctx: context | None = None, hbm_budget: int = 0, max_active: int = 64,
                 iters_per_step: int = 16, mixed: bool = True, rtol: float = 1e-8, inner_rtol: float = 1e-4):
        self.ctx = ctx or default_context()
        o = _lib.ServerOpts(int(hbm_budget), int(max_active), int(iters_per_step), _lib.F32 if mixed else _lib.F64,
                            0, float(rtol), float(inner_rtol))
        h = C.c_void_p()
        check(self.ctx._L.mtlg_server_create(self.ctx.h, C.byref(o), C.byref(h)), "server_create")
        self.h = h
        self.n = {}
        self.mixed = mixed

    def tune(self, requests, cache=None):
        """Sets the context's batched-pass knobs for requests like these
        ((A, b, solver, pc) tuples; measured on a sample once per class, then
        cached).  Call before the requests are submitted."""
        from . import autotune
        reqs = list(requests)
        if not reqs:
            return None
        kinds = {}
        for r in reqs:
            kinds[(r[2], r[3])] = kinds.get((r[2], r[3]), 0) + 1
        solver, pc = max(kinds, key=kinds.get)
        cache = cache or self.ctx.autotune or autotune.Cache()
        return autotune.tune_batch(self.ctx, [r[0] for r in reqs], solver, pc, self.mixed, cache=cache)[0]

    def submit(self, A, b, solver="cg", pc="ic_0", max_iter=2000) -> int:
        rp = np.ascontiguousarray(A.row_ptr, np.int64)
        ci = np.ascontiguousarray(A.col, np.int32)
        v = np.ascontiguousarray(A.val, np.float64)
        bb = np.ascontiguousarray(b, np.float64)
        rid = C.c_int64()
        check(self.ctx._L.mtlg_server_submit(self.h, A.n_rows, A.nnz, _p(rp), _p(ci), _p(v), _p(bb), _SOLVER[solver],
                                             _PC[pc], int(max_iter), C.byref(rid)), "server_submit")
        self.n[rid.value] = A.n_rows
        return rid.value

    def step(self):
        check(self.ctx._L.mtlg_server_step(self.h), "server_step")

    def poll(self, rid: int) -> Result | None:
        x = np.empty(self.n[rid])
        r = _lib.IterResult()
        st = self.ctx._L.mtlg_server_poll(self.h, rid, _p(x), C.byref(r))
        if st == _lib.PENDING:
            return None
        check(st, "server_poll")
        del self.n[rid]
        return _result(x, r)

    def cancel(self, rid: int):
        check(self.ctx._L.mtlg_server_cancel(self.h, rid), "server_cancel")
        self.n.pop(rid, None)

    def stats(self) -> dict:
        s = _lib.ServerStats()
        check(self.ctx._L.mtlg_server_stats_get(self.h, C.byref(s)), "server_stats")
        return {k: getattr(s, k) for k, _ in _lib.ServerStats._fields_}

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.ctx.h:
                self.ctx._L.mtlg_server_destroy(self.h)
        except Exception:
            pass


def run_open_loop(srv: server, requests, arrivals, timeout_s: float = 600.0):
    """Submits request i at arrival time arrivals[i] (seconds from start,
    host clock) while stepping the server; returns per-request latency
    (arrival -> result available on the host) and the results.

    requests: list of (A, b, solver, pc, max_iter)."""
    t0 = time.perf_counter()
    pending = {}
    lat = np.full(len(requests), np.nan)
    results = [None] * len(requests)
    nxt = 0
    while nxt < len(requests) or pending:
        now = time.perf_counter() - t0
        if now > timeout_s:
            break
        while nxt < len(requests) and arrivals[nxt] <= now:
            A, b, solver, pc, mi = requests[nxt]
            rid = srv.submit(A, b, solver, pc, mi)
            pending[rid] = nxt
            nxt += 1
        if pending:
            srv.step()
            for rid in list(pending):
                r = srv.poll(rid)
                if r is not None:
                    i = pending.pop(rid)
                    lat[i] = time.perf_counter() - t0 - arrivals[i]
                    results[i] = r
        elif nxt < len(requests):
            time.sleep(max(0.0, min(0.001, arrivals[nxt] - now)))
    wall = time.perf_counter() - t0
    done = np.isfinite(lat)
    return {"wall_s": wall, "completed": int(done.sum()), "solves_per_s": float(done.sum() / wall),
            "p50_s": float(np.percentile(lat[done], 50)) if done.any() else None,
            "p99_s": float(np.percentile(lat[done], 99)) if done.any() else None,
            "latency": lat, "results": results}
