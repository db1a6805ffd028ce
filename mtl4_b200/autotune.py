"""Launch-shape autotuner.

Measures the device-side knobs of the context (``mtlg_ctx_set_tuning``) on the
operator at hand and keeps the fastest setting.  Choices are cached in a JSON
file keyed by (GPU, kernel family, precision, n, nnz and the row-length
histogram in power-of-two buckets), so a repeated run -- or another matrix
with the same shape statistics -- reuses them without measuring.

Knobs:
  sweep_blocks   grid of the level-scheduled triangular sweeps (CTAs of 8 warps)
  sweep_sleep_ns back-off between polls of a dependency
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path

import numpy as np

DEFAULT_CACHE = Path(os.environ.get("MTL4_B200_TUNE_CACHE", Path.home() / ".cache" / "mtl4_b200" / "tune.json"))


def row_histogram(row_ptr: np.ndarray) -> list[int]:
    """Rows per power-of-two length bucket: [0], [1], [2,3], [4,7], ..."""
    lens = np.diff(np.asarray(row_ptr, dtype=np.int64))
    b = np.zeros(lens.shape, dtype=np.int64)
    nz = lens > 0
    b[nz] = np.floor(np.log2(lens[nz])).astype(np.int64) + 1
    return np.bincount(b, minlength=14).tolist()


def signature(gpu: str, family: str, dtype: str, A) -> str:
    hist = row_histogram(A.row_ptr)
    # coarse histogram (fractions rounded) so similar matrices share an entry
    tot = max(1, sum(hist))
    coarse = [round(h / tot, 2) for h in hist]
    return json.dumps([gpu, family, dtype, int(A.n_rows), int(A.nnz), coarse])


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


def sweep_candidates(sm_count: int):
    return [{"sweep_blocks": b, "sweep_sleep_ns": s}
            for b in (sm_count // 2, sm_count, sm_count + sm_count // 2, 2 * sm_count) for s in (0, 64)]


def tune_sweeps(ctx, A, P, dtype=np.float32, cache: Cache | None = None, reps: int = 3, gpu: str | None = None):
    """Chooses the sweep grid and back-off for preconditioner P of A (device
    objects from mtl4_b200.itl / .mtl; A also as problems.CSR for the key)."""
    from . import itl, mtl
    cache = cache or Cache()
    gpu = gpu or _gpu_name()
    key = signature(gpu, f"sweep:{type(P).__name__}", np.dtype(dtype).name, A)
    hit = cache.get(key)
    if hit:
        apply_settings(ctx, hit["choice"])
        return hit["choice"], True
    n = A.n_rows
    x = mtl.dense_vector(np.ones(n, dtype), dtype, ctx)
    y = mtl.dense_vector(n, dtype, ctx)

    def measure(c):
        apply_settings(ctx, c)
        itl.solve(P, x, y)
        ctx.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            itl.solve(P, x, y)
        ctx.synchronize()
        return (time.perf_counter() - t0) / reps

    choice, timings = best_of(sweep_candidates(ctx.get_tuning("sm_count")), measure)
    apply_settings(ctx, choice)
    cache.put(key, {"choice": choice, "timings": timings})
    return choice, False


def apply_settings(ctx, settings: dict):
    for k, v in settings.items():
        ctx.set_tuning(k, int(v))


def _gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown"
