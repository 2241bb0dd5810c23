"""Autotuner for rho1 plans: picks the tile shape and schedule of the grouped
launch by timing the candidates on the caller's own inputs.

Every candidate gives identical results (the tunings only change how batches
are cut into work items, how many CTAs share an SM and in which order the
persistent CTAs take the items), so the choice is purely by time.  Choices
are cached per (GPU, mode, batch geometry) in a JSON file.

    best = autotune.tune_rho1(plan, prob, run, mode=_lib.RHO1_FP64)
    # run() executes one rho1 step with plan on the current stream
"""

from __future__ import annotations

import hashlib
import json
import os

import numpy as np

from . import _lib

FP64_SPACE = [
    {"fp64_tile_points": 64, "fp64_ctas_per_sm": 0, "order": 2},
    {"fp64_tile_points": 64, "fp64_ctas_per_sm": 0, "order": 0},
    {"fp64_tile_points": 64, "fp64_ctas_per_sm": 1, "order": 2},
    {"fp64_tile_points": 64, "fp64_ctas_per_sm": 0, "order": 1},
    {"fp64_tile_points": 128, "fp64_ctas_per_sm": 0, "order": 2},
]
# (the work order is shared by both paths' lists; the FP64 search owns it)
SPLIT_SPACE = [
    {"split_tile_points": 128},
    {"split_tile_points": 96},
    {"split_tile_points": 64},
]


def space(mode: int) -> list[dict]:
    """Candidates per mode; the split-int8 mode has no shape tuning (its
    scratch budget changes how batches are grouped, not the speed)."""
    if mode == _lib.RHO1_SPLIT_I8:
        return [{}]
    return FP64_SPACE if mode == _lib.RHO1_FP64 else SPLIT_SPACE


def geometry_key(prob, mode: int, device_name: str = "") -> str:
    """Cache key: GPU name, mode, T and the batch shapes (n_compute, points)."""
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(prob.n_compute_c_batches, dtype=np.int32).tobytes())
    h.update(np.ascontiguousarray(prob.n_point_batches, dtype=np.int32).tobytes())
    return f"{device_name}|mode{mode}|T{prob.T}|{h.hexdigest()[:16]}"


def _time_ms(run, reps: int) -> float:
    import torch

    run()  # warm-up (and first-use set-up)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune_rho1(plan, prob, run, mode: int, reps: int = 2, cache_path: str | None = None) -> dict:
    """Times ``run`` under each candidate of ``space(mode)``, leaves the fastest
    applied to ``plan`` and returns {"choice", "ms", "timings", "cached"}."""
    import torch

    key = geometry_key(prob, mode, torch.cuda.get_device_name())
    cache = {}
    if cache_path and os.path.exists(cache_path):
        try:
            cache = json.load(open(cache_path))
        except (OSError, ValueError):
            cache = {}
    if key in cache:
        plan.set_tuning(**cache[key]["choice"])
        return dict(cache[key], cached=True)
    timings = []
    for cand in space(mode):
        plan.set_tuning(**cand)
        timings.append((_time_ms(run, reps), cand))
    ms, best = min(timings, key=lambda x: x[0])
    plan.set_tuning(**best)
    result = {"choice": best, "ms": ms, "timings": [{"ms": t, **c} for t, c in timings]}
    if cache_path:
        cache[key] = result
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1)
        os.replace(tmp, cache_path)
    return dict(result, cached=False)
