"""The autotuner's choice logic on the CPU (maccpic_b200/autotune.py), with a
stand-in run whose push and step times are a fixed table and a clock that
advances by them: it must time every variant's push, keep the fastest
within 10 % (at most three), sweep only the sort intervals the drift bound
allows, keep the pair with the shortest step, and remember it per device,
grid, density and precision in its cache (a broken cache file is ignored).
"""
import json

import pytest


class _Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


class _FakeRun:
    """push_ms[v]: regrouping push time of variant v; step_ms[(v, k)]: step
    time at sort interval k.  Every step advances the clock by its time."""

    def __init__(self, clock, push_ms, step_ms, kmax, nx=64, ny=32):
        class P:
            pass
        self.p = P()
        self.p.nx, self.p.ny, self.p.precision, self.p.device = nx, ny, 1, 0
        self.clock, self.push_ms, self.step_ms, self.kmax = clock, push_ms, step_ms, kmax
        self.v, self.k, self.timing = 0, 1, False
        self.timed = []
        self.steps_at = {}

    def num_variants(self):
        return len(self.push_ms)

    def set_variant(self, v):
        assert 0 <= v < len(self.push_ms)
        self.v = v

    def variant(self):
        return self.v, f"variant {self.v}"

    def set_sort_interval(self, k):
        assert 1 <= k <= self.kmax, k
        self.k = k

    def max_sort_interval(self):
        return self.kmax

    def reset_counters(self):
        self.timed = []

    def set_timing(self, on):
        self.timing = on

    def counters(self):
        return {"push_ms": sum(self.timed), "push_launches_timed": len(self.timed)}

    def step(self, n):
        for _ in range(n):
            if self.timing:
                self.timed.append(self.push_ms[self.v])
            self.clock.t += self.step_ms.get((self.v, self.k), 10.0) / 1e3
            self.steps_at[(self.v, self.k)] = self.steps_at.get((self.v, self.k), 0) + 1


@pytest.fixture
def clock(monkeypatch):
    import time
    c = _Clock()
    monkeypatch.setattr(time, "perf_counter", c)
    return c


def test_picks_the_fastest_pair_among_the_close_variants(clock, tmp_path):
    from maccpic_b200 import autotune
    push = [3.0, 2.9, 3.5, 3.15, 2.95]  # 1, 4, 0 within 10 % of 2.9 (3.15 too, but 4th)
    step = {(1, 1): 6.4, (1, 2): 6.2, (1, 3): 6.3, (4, 1): 6.5, (4, 2): 6.1, (4, 3): 6.25,
            (0, 1): 6.6, (0, 2): 6.35, (0, 3): 6.3}
    run = _FakeRun(clock, push, step, kmax=3)
    out = autotune.autotune(run, particles=64 * 32 * 16, cache=str(tmp_path / "c.json"))
    assert out["variant"] == 4 and out["sort_interval"] == 2
    assert (run.v, run.k) == (4, 2)
    assert sorted(int(v) for v in out["candidates"]) == [0, 1, 4]
    assert out["times_ms"] == pytest.approx(push)
    # intervals beyond the drift bound are never set (the stand-in asserts)
    assert set(out["interval_ms"]) == {"1", "2", "3"}
    assert not out["from_cache"]


def test_cache_per_device_grid_density_and_precision(clock, tmp_path):
    from maccpic_b200 import autotune
    cache = str(tmp_path / "c.json")
    push = [2.0, 3.0]
    step = {(0, 1): 5.0, (0, 2): 4.0}
    run = _FakeRun(clock, push, step, kmax=2)
    first = autotune.autotune(run, particles=64 * 32 * 16, cache=cache)
    assert (first["variant"], first["sort_interval"]) == (0, 2)
    table = json.load(open(cache))
    assert len(table) == 1 and "64x32" in next(iter(table))
    # the same key: from the cache, nothing timed
    run2 = _FakeRun(clock, push, step, kmax=2)
    again = autotune.autotune(run2, particles=64 * 32 * 16, cache=cache)
    assert again["from_cache"] and (run2.v, run2.k) == (0, 2) and not run2.steps_at
    # another density is another key
    run3 = _FakeRun(clock, push, step, kmax=2)
    autotune.autotune(run3, particles=64 * 32 * 8, cache=cache)
    assert run3.steps_at and len(json.load(open(cache))) == 2


def test_a_broken_cache_is_ignored(clock, tmp_path):
    from maccpic_b200 import autotune
    cache = tmp_path / "c.json"
    cache.write_text("{ not json")
    run = _FakeRun(clock, [2.0], {(0, 1): 5.0}, kmax=1)
    out = autotune.autotune(run, particles=64 * 32, cache=str(cache))
    assert out["variant"] == 0 and out["sort_interval"] == 1 and not out["from_cache"]
    assert json.load(open(cache))  # rewritten whole
