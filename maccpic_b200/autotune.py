"""Autotuner for the fast push: picks the kernel variant (cells per CTA and
CTAs per SM) by timing each one on the live state.

The variants are compiled into libem2g (em2g_num_variants); they compute the
same step, so tuning simply advances the run by a few steps per variant.
The particle sort is fused into the push and runs every step, so there is no
sort interval left to tune.  The winner is remembered per GPU model, grid,
particles per cell and precision in a small JSON cache.
"""
from __future__ import annotations

import json
import os

DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), ".autotune_cache.json")


def _key(run, particles: int) -> str:
    import torch
    dev = torch.cuda.get_device_name(run.p.device) if torch.cuda.is_available() else "cpu"
    ppc = particles / max(1, run.p.nx * run.p.ny)
    return f"{dev}|{run.p.nx}x{run.p.ny}|ppc{ppc:.1f}|prec{run.p.precision}"


def autotune(run, particles: int, steps: int = 2, warm: int = 1, cache: str | None = DEFAULT_CACHE,
             use_cache: bool = True) -> dict:
    """Time every variant on `run` (an Em2Gpu with its state loaded) and keep
    the fastest.  Returns {"variant", "name", "times_ms", "from_cache"}."""
    key = _key(run, particles)
    table = {}
    if cache and os.path.exists(cache):
        try:
            table = json.load(open(cache))
        except (OSError, ValueError):
            table = {}
    n = run.num_variants()
    if use_cache and key in table and 0 <= table[key]["variant"] < n:
        run.set_variant(table[key]["variant"])
        return {**table[key], "from_cache": True}
    times = []
    for v in range(n):
        run.set_variant(v)
        for _ in range(warm):
            run.step(1)
        run.reset_counters()
        run.set_timing(True)
        for _ in range(steps):
            run.step(1)
        c = run.counters()
        run.set_timing(False)
        times.append(c["push_ms"] / max(1, c["push_launches_timed"]))
    best = min(range(n), key=lambda v: times[v])
    run.set_variant(best)
    run.reset_counters()
    result = {"variant": best, "name": run.variant()[1], "times_ms": times}
    if cache:
        table[key] = result
        try:
            with open(cache, "w") as f:
                json.dump(table, f, indent=1)
        except OSError:
            pass
    return {**result, "from_cache": False}
