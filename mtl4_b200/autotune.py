"""Launch-shape autotuner.

Measures the device-side knobs of the context (``mtlg_ctx_set_tuning``) on the
operator at hand and keeps the fastest setting.  Choices are cached in a JSON
file keyed by (GPU, what is tuned, precision, n, nnz and the row-length
histogram in power-of-two buckets), so a repeated run -- or another matrix
with the same shape statistics -- reuses them without measuring.

Knobs and what measures them:
  spmv_kernel      standalone y = A x kernel: 0 auto, 1 stream tiles, 2 warp
                   tasks, 3 thread per row                     (tune_spmv)
  chunk_rows       rows per chunk of the chunked triangular sweeps; read when
                   a preconditioner is built, so each candidate rebuilds it
  sweep_cluster    CTAs per cluster of the chunked sweeps (0 automatic)
  grid_warps       compute warps per CTA of the grid sweeps (grid-stencil
                   factors; 0 automatic)                       (tune_pc)
  sweep_sleep_ns   back-off of the sweeps' dependency polls    (tune_pc)
  vec_ctas_per_sm  CTAs per SM of the vector passes of the Krylov loops
                                                               (tune_vec)
  sweep_blocks, sweep_sleep_ns   grid and back-off of the flat sweep kernel
                                                               (tune_sweeps)

The chunked-sweep and vector knobs are also tuned on a batch of systems
(tune_batch), measuring the batched solve itself.  Several knobs are searched
coordinate by coordinate: each knob in turn takes its fastest value with the
others held, each distinct setting measured once.

Wiring: with ``context.enable_autotune()`` the preconditioner constructors
(ilu_0, ic_0) apply the cached or freshly tuned sweep settings of their
operator class, the solvers apply the vector setting and mtl.mult the SpMV
kernel; serve.batch.solve(tune=True) and serve.server.tune(requests) tune the
batched passes.
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path

import numpy as np

DEFAULT_CACHE = Path(os.environ.get("MTL4_B200_TUNE_CACHE", Path.home() / ".cache" / "mtl4_b200" / "tune.json"))

SPMV_KERNELS = (0, 1, 2, 3)
VEC_CTAS = (1, 2, 4, 8)
SWEEP_CLUSTERS = (0, 1, 2, 4, 8, 16)
CHUNK_ROWS = (0, 4096, 8192, 16384, 32768)
GRID_WARPS = (0, 4, 8)


def row_histogram(row_ptr: np.ndarray) -> list[int]:
    """Rows per power-of-two length bucket: [0], [1], [2,3], [4,7], ..."""
    lens = np.diff(np.asarray(row_ptr, dtype=np.int64))
    b = np.zeros(lens.shape, dtype=np.int64)
    nz = lens > 0
    b[nz] = np.floor(np.log2(lens[nz])).astype(np.int64) + 1
    return np.bincount(b, minlength=14).tolist()


def _shape_key(n_rows: int, nnz: int, row_ptr) -> list:
    if row_ptr is None:
        return [int(n_rows), int(nnz), None]
    hist = row_histogram(row_ptr)
    # coarse histogram (fractions rounded) so similar matrices share an entry
    tot = max(1, sum(hist))
    return [int(n_rows), int(nnz), [round(h / tot, 2) for h in hist]]


def signature(gpu: str, family: str, dtype: str, A) -> str:
    """Cache key of operator A (problems.CSR, or anything with n_rows / nnz
    and, optionally, row_ptr)."""
    return json.dumps([gpu, family, dtype] + _shape_key(A.n_rows, A.nnz, getattr(A, "row_ptr", None)))


def batch_signature(gpu: str, family: str, dtype: str, systems) -> str:
    """Cache key of a set of systems: count, total rows and entries, and the
    coarse row-length histogram of all of them together."""
    hist = np.zeros(14, dtype=np.int64)
    rows = nnz = 0
    for A in systems:
        h = row_histogram(A.row_ptr)
        hist[:len(h)] += np.asarray(h[:14])
        rows += int(A.n_rows)
        nnz += int(A.nnz)
    tot = max(1, int(hist.sum()))
    return json.dumps([gpu, family, dtype, len(systems), rows, nnz, [round(int(h) / tot, 2) for h in hist]])


class Cache:
    def __init__(self, path: Path | str = DEFAULT_CACHE):
        self.path = Path(path)
        self.data: dict[str, dict] = {}
        if self.path.exists():
            try:
                self.data = json.loads(self.path.read_text())
            except Exception:
                self.data = {}

    def get(self, key: str):
        return self.data.get(key)

    def put(self, key: str, value: dict):
        self.data[key] = value
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            tmp = self.path.with_suffix(".tmp")
            tmp.write_text(json.dumps(self.data, indent=1, sort_keys=True))
            tmp.replace(self.path)
        except OSError:
            pass


def best_of(candidates, measure):
    """Returns (best candidate, {candidate: seconds}) with measure(candidate)
    -> seconds (smallest wins; ties keep the earlier candidate)."""
    timings = {}
    best, best_t = None, float("inf")
    for c in candidates:
        t = measure(c)
        timings[json.dumps(c, sort_keys=True)] = t
        if t < best_t:
            best, best_t = c, t
    return best, timings


def coordinate_search(space: dict, start: dict, measure):
    """Knob by knob (in the order of `space`): every value of the knob with
    the others at their current best; the fastest value is kept before the
    next knob.  A setting already measured is not measured again.  Returns
    (best setting, {setting: seconds})."""
    timings: dict[str, float] = {}
    best = dict(start)

    def timed(c):
        k = json.dumps(c, sort_keys=True)
        if k not in timings:
            timings[k] = measure(dict(c))
        return timings[k]

    best_t = timed(best)
    for knob, values in space.items():
        for v in values:
            c = dict(best)
            c[knob] = v
            t = timed(c)
            if t < best_t:
                best, best_t = c, t
    return best, timings


def sweep_candidates(sm_count: int):
    return [{"sweep_blocks": b, "sweep_sleep_ns": s}
            for b in (sm_count // 2, sm_count, sm_count + sm_count // 2, 2 * sm_count) for s in (0, 64)]


def apply_settings(ctx, settings: dict):
    for k, v in settings.items():
        ctx.set_tuning(k, int(v))


def current_settings(ctx, knobs) -> dict:
    return {k: int(ctx.get_tuning(k)) for k in knobs}


def _gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown"


def _timed(fn, reps: int, ctx) -> float:
    fn()
    ctx.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    ctx.synchronize()
    return (time.perf_counter() - t0) / reps


def _cached(cache, key, ctx):
    hit = cache.get(key)
    if hit:
        apply_settings(ctx, hit["choice"])
        return hit["choice"]
    return None


def _host_shape(Ad):
    """(n_rows, nnz, host row_ptr or None) of a device compressed2D."""
    return Ad.shape[0], Ad.nnz, getattr(Ad, "host_row_ptr", None)


class _Shape:
    def __init__(self, n_rows, nnz, row_ptr):
        self.n_rows, self.nnz, self.row_ptr = n_rows, nnz, row_ptr


def tune_spmv(ctx, Ad, cache: Cache | None = None, reps: int = 5, gpu: str | None = None):
    """Chooses the standalone SpMV kernel for device matrix Ad (FP64 x)."""
    from . import mtl
    cache = cache or Cache()
    key = signature(gpu or _gpu_name(), "spmv", "float64", _Shape(*_host_shape(Ad)))
    hit = _cached(cache, key, ctx)
    if hit is not None:
        return hit, True
    x = mtl.dense_vector(np.ones(Ad.shape[1]), np.float64, ctx)
    y = mtl.dense_vector(Ad.shape[0], np.float64, ctx)

    def measure(c):
        apply_settings(ctx, c)
        return _timed(lambda: mtl.mult(Ad, x, y, tune=False), reps, ctx)

    choice, timings = best_of([{"spmv_kernel": k} for k in SPMV_KERNELS], measure)
    apply_settings(ctx, choice)
    cache.put(key, {"choice": choice, "timings": timings})
    return choice, False


def tune_pc(ctx, Ad, kind: str, value=np.float32, cache: Cache | None = None, reps: int = 3,
            gpu: str | None = None, space: dict | None = None):
    """Chooses chunk_rows and sweep_cluster for preconditioner `kind`
    ("ilu_0" or "ic_0", stored in `value`) of device matrix Ad by timing its
    apply; each chunk_rows candidate builds the preconditioner anew.  A
    preconditioner swept by the grid kernel (grid-stencil factors) tunes
    grid_warps instead."""
    from . import itl, mtl
    cache = cache or Cache()
    dt = np.dtype(value)
    key = signature(gpu or _gpu_name(), f"pc:{kind}", dt.name, _Shape(*_host_shape(Ad)))
    hit = _cached(cache, key, ctx)
    if hit is not None:
        return hit, True
    n = Ad.shape[0]
    x = mtl.dense_vector(np.ones(n, dt), dt, ctx)
    y = mtl.dense_vector(n, dt, ctx)
    built = {}
    cls = getattr(itl.pc, kind)
    if space is None:
        probe = cls(Ad, dt, tune=False)
        grid = probe.sweep_plan(dt).get("kernel") == "grid"
        del probe
        space = {"grid_warps": GRID_WARPS} if grid else {"chunk_rows": CHUNK_ROWS, "sweep_cluster": SWEEP_CLUSTERS}

    def measure(c):
        apply_settings(ctx, c)
        cr = c.get("chunk_rows", 0)
        if cr not in built:
            built.clear()   # one candidate preconditioner on the device at a time
            built[cr] = cls(Ad, dt, tune=False)
        P = built[cr]
        return _timed(lambda: itl.solve(P, x, y), reps, ctx)

    start = {k: 0 for k in space}   # every knob of the space at its default (0)
    choice, timings = coordinate_search(space, start, measure)
    built.clear()
    apply_settings(ctx, choice)
    cache.put(key, {"choice": choice, "timings": timings})
    return choice, False


def tune_vec(ctx, Ad, value=np.float64, cache: Cache | None = None, iters: int = 30, reps: int = 2,
             gpu: str | None = None):
    """Chooses vec_ctas_per_sm by timing `iters` unpreconditioned CG
    iterations on Ad (the fused SpMV+dot and vector passes of the loop)."""
    from . import itl, mtl
    cache = cache or Cache()
    dt = np.dtype(value)
    key = signature(gpu or _gpu_name(), "vec", dt.name, _Shape(*_host_shape(Ad)))
    hit = _cached(cache, key, ctx)
    if hit is not None:
        return hit, True
    n = Ad.shape[0]
    b = mtl.dense_vector(np.ones(n), np.float64, ctx)
    x = mtl.dense_vector(n, np.float64, ctx)

    def run():
        x.fill(0.0)
        it = itl.basic_iteration(b, iters, 1e-300)
        itl.cg(Ad, x, b, None, it, tune=False)

    def measure(c):
        apply_settings(ctx, c)
        return _timed(run, reps, ctx)

    choice, timings = best_of([{"vec_ctas_per_sm": v} for v in VEC_CTAS], measure)
    apply_settings(ctx, choice)
    cache.put(key, {"choice": choice, "timings": timings})
    return choice, False


def tune_batch(ctx, systems, solver: str = "cg", pc: str = "ic_0", mixed: bool = False, iters: int = 30,
               cache: Cache | None = None, max_systems: int = 64, reps: int = 1, gpu: str | None = None,
               space: dict | None = None):
    """Chooses vec_ctas_per_sm, sweep_cluster and chunk_rows for batched
    solves of `systems` (problems.CSR; the right-hand sides are ones) by
    timing `iters` iterations of a batch of at most `max_systems` of them."""
    from . import serve
    cache = cache or Cache()
    sample = list(systems)[:max_systems]
    fam = f"batch:{solver}:{pc}:{'mixed' if mixed else 'fp64'}"
    key = batch_signature(gpu or _gpu_name(), fam, "float32" if mixed else "float64", sample)
    hit = _cached(cache, key, ctx)
    if hit is not None:
        return hit, True
    if space is None:
        space = {"vec_ctas_per_sm": VEC_CTAS}
        if pc in ("ilu_0", "ic_0"):
            space["grid_warps"] = GRID_WARPS
            space["sweep_cluster"] = SWEEP_CLUSTERS
            space["chunk_rows"] = CHUNK_ROWS
    start = {k: 0 for k in space}
    start["vec_ctas_per_sm"] = int(ctx.get_tuning("vec_ctas_per_sm"))

    def measure(c):
        apply_settings(ctx, c)

        def run():
            bt = serve.batch(ctx)
            for A in sample:
                bt.add(A, np.ones(A.n_rows), solver, pc, max_iter=iters, rtol=1e-300)
            bt.solve(mixed=mixed, rtol=1e-300, max_outer=1, max_inner=iters)
            del bt
        return _timed(run, reps, ctx)

    choice, timings = coordinate_search(space, start, measure)
    apply_settings(ctx, choice)
    cache.put(key, {"choice": choice, "timings": timings})
    return choice, False


def tune_sweeps(ctx, A, P, dtype=np.float32, cache: Cache | None = None, reps: int = 3, gpu: str | None = None):
    """Chooses the flat sweep grid and back-off for preconditioner P of A
    (device objects from mtl4_b200.itl / .mtl; A also as problems.CSR for the
    key)."""
    from . import itl, mtl
    cache = cache or Cache()
    gpu = gpu or _gpu_name()
    key = signature(gpu, f"sweep:{type(P).__name__}", np.dtype(dtype).name, A)
    hit = _cached(cache, key, ctx)
    if hit is not None:
        return hit, True
    n = A.n_rows
    x = mtl.dense_vector(np.ones(n, dtype), dtype, ctx)
    y = mtl.dense_vector(n, dtype, ctx)

    def measure(c):
        apply_settings(ctx, c)
        return _timed(lambda: itl.solve(P, x, y), reps, ctx)

    choice, timings = best_of(sweep_candidates(ctx.get_tuning("sm_count")), measure)
    apply_settings(ctx, choice)
    cache.put(key, {"choice": choice, "timings": timings})
    return choice, False
