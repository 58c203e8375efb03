"""Autotuner for a plan's launch knobs (row-split threshold, claim sizes, kernel
variant, team size, L2 retention).

``autotune(plan, op, x, y)`` times each candidate configuration on the actual
operands with CUDA events (after warm-up, each candidate the median of a few
repetitions), leaves the plan tuned to the fastest and returns the timings.
Results are remembered per (plan, op, columns, dtypes), so a second call with
the same shapes only re-applies the winner.  Re-laying out a plan (a new
chunk size or hot set) is host work: tune before capturing CUDA graphs.
"""
from __future__ import annotations

import itertools
import statistics

import torch

__all__ = ["autotune", "DEFAULT_SPACE"]

DEFAULT_SPACE = {
    "chunk_nnz": [128, 256, 512],
    "rows_per_claim": [2, 4, 8],
    "variant": ["auto", "register"],
    "hot_rows": [0, 65536],
}

_cache = {}


def _time(fn, reps, iters):
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(iters):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) / iters)
    return statistics.median(ts)


def autotune(plan, op, x, y, space=None, reps=3, iters=5, warmup=2):
    """Tunes ``plan`` for y <- op(A) x; returns [(config, ms)] sorted by time."""
    key = (id(plan), op, x.shape[1], x.dtype, y.dtype)
    if key in _cache:
        best = _cache[key][0][0]
        plan.tune(**best)
        return _cache[key]
    space = dict(DEFAULT_SPACE if space is None else space)
    names = list(space)
    results = []
    for values in itertools.product(*(space[k] for k in names)):
        cfg = dict(zip(names, values))
        plan.tune(**cfg)
        fn = lambda: plan.matmul(op, x, y)  # noqa: E731
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        results.append((cfg, _time(fn, reps, iters)))
    results.sort(key=lambda r: r[1])
    plan.tune(**results[0][0])
    plan.check_device()
    _cache[key] = results
    return results
