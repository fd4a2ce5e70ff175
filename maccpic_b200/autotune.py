"""Autotuner for the fast push: picks the kernel variant (cells per CTA =
the tile width, and CTAs per SM, which sets the particles in flight per SM)
and the sort interval by timing them on the live state.

The variants are compiled into libem2g (em2g_num_variants); they compute the
same step, so tuning simply advances the run by a few steps per candidate.
The sort interval trades the regrouping work of the push (per-cell write
positions, the scan of the cell counts) against the growing share of
particles outside their group cell, which deposit with atomics: the
interval is timed as whole steps over full regrouping cycles.  The winner is
remembered per GPU model, grid, particles per cell and precision in a small
JSON cache.
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


def _step_ms(run, k: int, cycles: int) -> float:
    """Mean wall time of a step at sort interval k over whole cycles."""
    import time
    run.set_sort_interval(k)
    # untimed: two cycles, so that an ensemble has captured the graph of
    # every kind of step (in place or regrouping, either buffer and count
    # parity) before the timing
    run.step(2 * k)
    n = k * cycles
    t = time.perf_counter()
    run.step(n)
    return (time.perf_counter() - t) * 1e3 / n


def autotune(run, particles: int, steps: int = 2, warm: int = 1, cache: str | None = DEFAULT_CACHE,
             use_cache: bool = True, intervals=None) -> dict:
    """Time every variant's regrouping push on `run` (an Em2Gpu with its state
    loaded), then time whole steps at every admissible sort interval for the
    fastest few, and keep the best (variant, interval).  Returns {"variant",
    "name", "times_ms", "sort_interval", "interval_ms" (of the kept variant),
    "candidates", "from_cache"}."""
    key = _key(run, particles)
    table = {}
    if cache and os.path.exists(cache):
        try:
            table = json.load(open(cache))
        except (OSError, ValueError):
            table = {}
    n = run.num_variants()
    if (use_cache and key in table and 0 <= table[key]["variant"] < n
            and "sort_interval" in table[key]):
        run.set_variant(table[key]["variant"])
        run.set_sort_interval(table[key]["sort_interval"])
        return {**table[key], "from_cache": True}
    run.set_sort_interval(1)
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
    # the variants within 10 % of the fastest regrouping push (at most 3) are
    # timed as whole steps at every admissible interval: between regroupings
    # the pushes run in place, and the variants' order can differ there
    order = sorted(range(n), key=lambda v: times[v])
    cands = [v for v in order[:3] if times[v] <= 1.1 * times[order[0]]]
    kmax = run.max_sort_interval()
    if intervals is None:
        intervals = sorted({k for k in (1, 2, 3, 4, 6, kmax) if 1 <= k <= kmax})
    sweep = {}
    for v in cands:
        run.set_variant(v)
        sweep[v] = {k: _step_ms(run, k, cycles=max(1, 12 // k)) for k in intervals}
    best, k_best = min(((v, k) for v in cands for k in intervals), key=lambda vk: sweep[vk[0]][vk[1]])
    run.set_variant(best)
    run.set_sort_interval(k_best)
    interval_ms = sweep[best]
    run.reset_counters()
    result = {"variant": best, "name": run.variant()[1], "times_ms": times,
              "sort_interval": k_best, "interval_ms": {str(k): v for k, v in interval_ms.items()},
              "candidates": {str(v): {str(k): t for k, t in sweep[v].items()} for v in cands}}
    if cache:
        table[key] = result
        try:
            with open(cache, "w") as f:
                json.dump(table, f, indent=1)
        except OSError:
            pass
    return {**result, "from_cache": False}


def autotune_ensemble(ens, steps: int = 2, warm: int = 1, intervals=None) -> dict:
    """Time every push variant on an ensemble (its current state, a few
    graph-launched steps each; every step advances the runs), then time the
    fastest few at every sort interval the drift bound allows and keep the
    best pair.  Returns {"variant", "times_ms", "sort_interval",
    "interval_ms", "candidates"}: mean wall time of a step per variant and
    per interval."""
    import time
    import torch
    ens.set_sort_interval(1)
    times = []
    for v in range(ens.num_variants()):
        ens.set_variant(v)
        ens.step(warm)
        torch.cuda.synchronize()
        t = time.perf_counter()
        ens.step(steps)
        torch.cuda.synchronize()
        times.append((time.perf_counter() - t) * 1e3 / steps)
    # as autotune: the fastest few (within 10 %, at most 3) at every interval
    order = sorted(range(len(times)), key=lambda v: times[v])
    cands = [v for v in order[:3] if times[v] <= 1.1 * times[order[0]]]
    kmax = ens.max_sort_interval()
    if intervals is None:
        intervals = sorted({k for k in (1, 2, 3, 4, 6, kmax) if 1 <= k <= kmax})
    sweep = {}
    for v in cands:
        ens.set_variant(v)
        sweep[v] = {k: _step_ms(ens, k, cycles=max(1, 6 // k)) for k in intervals}
    best, k_best = min(((v, k) for v in cands for k in intervals), key=lambda vk: sweep[vk[0]][vk[1]])
    ens.set_variant(best)
    ens.set_sort_interval(k_best)
    return {"variant": best, "times_ms": times, "sort_interval": k_best,
            "interval_ms": {str(k): v for k, v in sweep[best].items()},
            "candidates": {str(v): {str(k): t for k, t in sweep[v].items()} for v in cands}}
