#!/usr/bin/env python
"""Benchmark of the sparse-solve hot path on B200 (one JSON line on rank 0).

Workload (one step = one solve): BiCGSTAB + ILU(0) on the 3D 7-point
convection-diffusion operator on a 128^3 grid (2,097,152 unknowns,
14,581,760 entries, beta = (0.5, 0.3, 0.2), h = 1/129), b = A x_true with
x_true ~ U(-1,1) seed 1, to relative residual <= 1e-8.  ``value`` is the
mixed-precision path (FP32 inner BiCGSTAB with an FP32-stored ILU(0)
factorized in FP64, wrapped in FP64 iterative refinement); the plain FP64
path runs on the same inputs and is reported beside it.  The standalone SpMV
on the power-law CSR (4,194,304 rows) is reported as ``spmv``.

Inputs are larger than L2 (126 MB): A in FP64 + FP32 and the factors hold
~400 MB, touched every iteration, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun, one process per GPU) every rank solves its own replica
(no collective on the data path); value = all ranks' solves / max-over-ranks
time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "solves/s at relres<=1e-8, mixed vs plain FP64 on B200; SpMV %HBM; p99 latency"
WORKLOAD = ("BiCGSTAB+ILU(0) on 128^3 7-point convection-diffusion (2,097,152 unknowns, 14,581,760 nnz, "
            "beta=(0.5,0.3,0.2), h=1/129), b=A*x_true seed 1, relres<=1e-8")
PEAKS = ROOT / "MEASURED_PEAKS.json"
# DRAM bytes (read + write) of one FP32 ILU(0) apply (L and U k_sweep_chunk
# launches) from ncu on this workload; see profiles/k_sweep_chunk_ilu0_convdiff128_f32.md
TRAFFIC_PER_APPLY = 210_680_000   # 105.1 MB (L) + 105.5 MB (U)
FALLBACK_HBM = 6650.0


def hbm_peak():
    try:
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ distributed
def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def dist_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ------------------------------------------------------------------ reference arm
def cpu_reference_solve(A, b, threads_omp=True):
    """MTL4's own BiCGSTAB + ILU(0) (oracle/_ref, unchanged reference
    headers), FP64, on the host cores.  Returns (seconds, result)."""
    from oracle import oracle as O
    R = O.RefMatrix(A, omp=threads_omp)
    r = R.solve(b, "bicgstab", "ilu_0", max_iter=2000, rtol=1e-8)
    return r["solve_s"] + r["setup_s"], r, R.L.mtlref_openmp_threads()


def run_reference(args, rank, world):
    if rank != 0:
        return
    from mtl4_b200 import problems as P
    from oracle import oracle as O
    if not O.ref_available(omp=True):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmtlref_omp.so not built"}))
        return
    A, b, _ = P.config2_solve(128)
    times, res, thr = [], None, 1
    for i in range(args.warmup + args.steps):
        s, res, thr = cpu_reference_solve(A, b)
        if i >= args.warmup:
            times.append(s)
    sec = float(np.mean(times))
    val = 1.0 / sec
    line = {"metric": METRIC, "value": val, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": WORKLOAD, "solver": "itl::bicgstab + itl::pc::ilu_0<compressed2D<double>>",
                       "iterations": res["iterations"], "relres": res["relresid"]},
            "cpu_baseline": {"value": val, "unit": "solves/s", "cores": thr, "kind": "reference",
                             "sample": f"{args.steps} full solves (setup + solve), OpenMP build, {thr} threads"},
            "e2e": {"value": val, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ batched and served samples
def batch_and_serve(ctx, n_batch=64, n_req=24, rates=(1.0, 2.0, 4.0)):
    """Bounded samples of the batched and the served workloads: every 16th
    of the 1,024 uneven systems (same size distribution) solved as one batch
    (FP64, and FP32 inner / FP64 refinement), and the first n_req requests of
    the 20,000-request stream under open-loop Poisson arrivals at each of a
    sweep of rates (p50 / p99 of arrival -> result on the host, setup
    included, beside the completed solves/s).  The inner FP32 solves stop at
    1e-5 (fewer restarts than at 1e-4 on these operators)."""
    import time as _t
    from mtl4_b200 import problems as P
    from mtl4_b200 import serve
    out = {}
    specs = P.batch_specs(1024)[::1024 // n_batch]
    systems = [sp.build() for sp in specs]
    rhs = [P.random_rhs(A.n_rows, sp.seed) for sp, A in zip(specs, systems)]
    rows = int(sum(A.n_rows for A in systems))
    for mixed in (False, True):
        B = serve.batch(ctx)
        for sp, A, b in zip(specs, systems, rhs):
            B.add(A, b, sp.solver, sp.pc, max_iter=3000, rtol=1e-8)
        ctx.synchronize()
        t0 = _t.perf_counter()
        B.solve(mixed=mixed, rtol=1e-8, inner_rtol=1e-5)
        ctx.synchronize()
        t1 = _t.perf_counter()
        B.solve(mixed=mixed, rtol=1e-8, inner_rtol=1e-5)
        ctx.synchronize()
        t2 = _t.perf_counter()
        res = [B.result(i) for i in range(len(systems))]
        ok = sum(1 for r in res if r.error_code == 0)
        worst = max(float(np.linalg.norm(A.matvec(r.x) - b) / np.linalg.norm(b))
                    for A, b, r in zip(systems, rhs, res))
        out["mixed" if mixed else "fp64"] = {
            "systems": len(systems), "rows": rows, "converged": ok, "worst_relres": worst,
            "solve_s": t2 - t1, "solves_per_s": len(systems) / (t2 - t1), "first_solve_with_setup_s": t1 - t0}
        del B
    rspecs = P.request_specs(20000)[:n_req]
    reqs = []
    for sp in rspecs:
        A = sp.build()
        reqs.append((A, P.random_rhs(A.n_rows, sp.seed), sp.solver, sp.pc, 3000))
    out["served"] = []
    for rate in rates:
        arrivals = P.poisson_arrivals(n_req, rate)
        srv = serve.server(ctx, max_active=64, iters_per_step=16, mixed=True, rtol=1e-8, inner_rtol=1e-5)
        r = serve.run_open_loop(srv, reqs, arrivals, timeout_s=240.0)
        ok = sum(1 for x in r["results"] if x is not None and x.error_code == 0)
        out["served"].append({"requests": n_req, "rate_per_s": rate, "completed": r["completed"], "converged": ok,
                              "rows": int(sum(q[0].n_rows for q in reqs)), "wall_s": r["wall_s"],
                              "solves_per_s": r["solves_per_s"], "p50_s": r["p50_s"], "p99_s": r["p99_s"],
                              "clock": "host, arrival -> result available (setup included)"})
        del srv
    return out


# ------------------------------------------------------------------ profiling cases
def run_kernel_case(args):
    """One kernel on its bench case, `reps` times (no timing output): the
    command line the committed ncu summaries under profiles/ were made with."""
    from mtl4_b200 import itl, mtl
    from mtl4_b200 import problems as P
    ctx = mtl.context(0)
    if args.kernel in ("spmv_powerlaw", "spmv_stencil"):
        A = P.config2_spmv() if args.kernel == "spmv_powerlaw" else P.config2_solve(128)[0]
        Ad = mtl.compressed2D.from_problem(A, ctx)
        x = mtl.dense_vector(np.random.default_rng(0).standard_normal(A.n_rows), np.float64, ctx)
        y = mtl.dense_vector(A.n_rows, np.float64, ctx)
        for _ in range(args.reps):
            mtl.mult(Ad, x, y)
    elif args.kernel == "sweep_ilu0":
        A, b, _ = P.config2_solve(128)
        Ad = mtl.compressed2D.from_problem(A, ctx)
        Pc = itl.pc.ilu_0(Ad, np.float32)
        bf = mtl.dense_vector(b.astype(np.float32), np.float32, ctx)
        yf = mtl.dense_vector(A.n_rows, np.float32, ctx)
        for _ in range(args.reps):
            itl.solve(Pc, bf, yf)
    else:
        A, b, _ = P.config2_solve(128)
        Ad = mtl.compressed2D.from_problem(A, ctx)
        Pc = itl.pc.ilu_0(Ad, np.float32)
        bd = mtl.dense_vector(b, np.float64, ctx)
        for _ in range(args.reps):
            x = mtl.dense_vector(A.n_rows, np.float64, ctx)
            itl.refine("bicgstab", Ad, x, bd, Pc, rtol=1e-8, inner_rtol=1e-4)
    ctx.synchronize()
    print(json.dumps({"kernel": args.kernel, "reps": args.reps, "launches": ctx.kernel_launches()}))


# ------------------------------------------------------------------ GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mtl4_b200", choices=["mtl4_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the batched / served samples")
    ap.add_argument("--kernel", choices=["spmv_powerlaw", "spmv_stencil", "sweep_ilu0", "solve_mixed"],
                    help="run one kernel on its bench case a few times and exit (for profilers)")
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup) if args.impl != "reference" else args.warmup
    if args.kernel:
        run_kernel_case(args)
        return
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    from mtl4_b200 import _lib, itl, mtl
    from mtl4_b200 import problems as P

    torch.cuda.set_device(local)
    # a dedicated (non-default) stream: kernels and timing events share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = mtl.context(local)
    ctx.set_stream(stream.cuda_stream)
    mtl._DEFAULT[local] = ctx

    A, b, x_true = P.config2_solve(128)
    n = A.n_rows
    Ad = mtl.compressed2D.from_problem(A, ctx)
    P64 = itl.pc.ilu_0(Ad, np.float64)
    P32 = itl.pc.ilu_0(Ad, np.float32)
    b_pin = torch.from_numpy(b).pin_memory()
    x_pin = torch.empty(n, dtype=torch.float64).pin_memory()
    bd = mtl.dense_vector(b, np.float64, ctx)
    xd = mtl.dense_vector(n, np.float64, ctx)
    L = ctx._L

    def solve_mixed():
        xd.fill(0.0)
        return itl.refine("bicgstab", Ad, xd, bd, P32, rtol=1e-8, inner_rtol=1e-4, max_outer=20, max_inner=2000)

    def solve_fp64():
        xd.fill(0.0)
        it = itl.basic_iteration(bd, 2000, 1e-8)
        itl.bicgstab(Ad, xd, bd, P64, it)
        return it

    def timed(fn, k, w):
        for _ in range(w):
            it = fn()
        dist_barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.kernel_launches()
        e0.record(stream)
        for _ in range(k):
            it = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        dist_barrier(world)
        sec = e0.elapsed_time(e1) * 1e-3
        return dist_max(sec, world), it, ctx.kernel_launches() - l0

    with ClockSampler(local) as clk:
        t_mixed, it_mixed, launches = timed(solve_mixed, args.steps, args.warmup)
    clocks = clk.summary()
    x_mixed = xd.numpy()
    relres_mixed = float(np.linalg.norm(A.matvec(x_mixed) - b) / np.linalg.norm(b))
    t_fp64, it_fp64, _ = timed(solve_fp64, max(2, args.steps // 2), 1)
    x_fp64 = xd.numpy()
    relres_fp64 = float(np.linalg.norm(A.matvec(x_fp64) - b) / np.linalg.norm(b))
    k64 = max(2, args.steps // 2)

    # end to end through the public API with host buffers (pinned): upload b,
    # solve, read x back, every step
    def e2e_step():
        L.mtlg_vec_upload(bd.h, _lib.C.c_void_p(b_pin.data_ptr()), n)
        it = solve_mixed()
        L.mtlg_vec_download(xd.h, _lib.C.c_void_p(x_pin.data_ptr()), n)
        return it
    t_e2e, _, _ = timed(e2e_step, args.steps, 1)

    # error against an FP64 oracle-quality solve (tight plain FP64 GPU solve)
    xd.fill(0.0)
    it_t = itl.basic_iteration(bd, 4000, 1e-13)
    itl.bicgstab(Ad, xd, bd, P64, it_t)
    x_tight = xd.numpy()
    err_vs_fp64 = float(np.abs(x_mixed - x_tight).max() / np.abs(x_tight).max())

    # dominant kernel: the chunked triangular sweeps of the FP32 ILU(0)
    # apply (k_sweep_chunk, L then U), timed with events on the launching
    # stream; the applies are queued back to back (pc_apply_sync = 0), then
    # one synchronous apply reports any expired device wait
    bf = mtl.dense_vector(b.astype(np.float32), np.float32, ctx)
    yf = mtl.dense_vector(n, np.float32, ctx)
    for _ in range(3):
        itl.solve(P32, bf, yf)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    ctx.set_tuning("pc_apply_sync", 0)
    e0.record(stream)
    for _ in range(reps):
        itl.solve(P32, bf, yf)
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.set_tuning("pc_apply_sync", 1)
    itl.solve(P32, bf, yf)
    apply_s = e0.elapsed_time(e1) * 1e-3 / reps
    lev_L, lev_U = P32.levels()
    plan = P32.sweep_plan(np.float32)
    Lr, Lc, Lv = P32.factor("L")
    Ur, Uc, Uv = P32.factor("U")
    # algorithmic bytes of one apply (two sweeps), FP32 values, int32 indices:
    # factor values + columns, row pointers, row map and diagonal per
    # (level-ordered) row, right-hand side read, result written, and the
    # temporary written and re-armed once each
    nnz_off = len(Lv) + (len(Uv) - n)
    bytes_apply = 8 * nnz_off + 2 * 12 * n + 4 * n * 4
    peak, peak_kind = hbm_peak()
    sweep_gbs = bytes_apply / apply_s / 1e9

    # SpMV on the power-law CSR
    Q = P.config2_spmv()
    Qd = mtl.compressed2D.from_problem(Q, ctx)
    xq = mtl.dense_vector(np.random.default_rng(0).standard_normal(Q.n_rows), np.float64, ctx)
    yq = mtl.dense_vector(Q.n_rows, np.float64, ctx)
    for _ in range(3):
        mtl.mult(Qd, xq, yq)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        mtl.mult(Qd, xq, yq)
    e1.record(stream)
    torch.cuda.synchronize()
    spmv_s = e0.elapsed_time(e1) * 1e-3 / reps
    spmv_bytes = 12 * Q.nnz + 4 * (Q.n_rows + 1) + 8 * Q.n_rows + 8 * Q.n_rows
    spmv_gbs = spmv_bytes / spmv_s / 1e9

    if rank != 0:
        return
    value = world * args.steps / t_mixed
    v64 = world * k64 / t_fp64
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_mixed / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded generators)",
        "config": {"workload": WORKLOAD, "precision": "FP32 inner BiCGSTAB + FP32-stored ILU(0), FP64 refinement",
                   "l2": "inputs larger than L2 (~400 MB touched per iteration); no flush",
                   "parallelism": f"replicas x{world}"},
        "mixed": {"solves_per_s": value, "iterations": it_mixed.iterations(), "outer": it_mixed.outer,
                  "relres": relres_mixed, "err_vs_fp64_solve": err_vs_fp64},
        "fp64": {"solves_per_s": v64, "iterations": it_fp64.iterations(), "relres": relres_fp64},
        "mixed_over_fp64": value / v64,
        "spmv": {"matrix": f"power-law CSR {Q.n_rows} rows, {Q.nnz} nnz", "us": spmv_s * 1e6, "GBs": spmv_gbs,
                 "frac_measured_peak": spmv_gbs / peak, "frac_8TBs_nominal": spmv_gbs / 8000.0},
        "roofline": {"kernel": "k_sweep_chunk<float,float> (ILU(0) L and U sweeps, one apply)", "bound": "hbm",
                     "achieved": sweep_gbs, "peak": peak, "unit": "GB/s", "frac": sweep_gbs / peak,
                     "peak_kind": peak_kind, "traffic": TRAFFIC_PER_APPLY,
                     "algorithmic_bytes_per_apply": bytes_apply, "apply_us": apply_s * 1e6,
                     "levels": lev_L + lev_U, "ns_per_level": apply_s * 1e9 / (lev_L + lev_U),
                     "note": "dependency-latency bound: one level of the L or U chain per step",
                     "plan": plan},
        "e2e": {"value": world * args.steps / t_e2e, "unit": "solves/s", "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 8 * n},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if not args.no_serve:
        line["batched_and_served"] = batch_and_serve(ctx)
    if not args.no_cpu_baseline and world == 1:
        try:
            from oracle import oracle as O
            if O.ref_available(omp=True):
                s, r, thr = cpu_reference_solve(A, b)
                line["cpu_baseline"] = {"value": 1.0 / s, "unit": "solves/s", "cores": thr, "kind": "reference",
                                        "sample": "1 full solve (ILU(0) setup + BiCGSTAB) of the same system, "
                                                  f"OpenMP build, {r['iterations']} iterations"}
        except Exception as e:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
