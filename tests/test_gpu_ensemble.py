"""Ensembles (maccpic_b200/ensemble.py, em2g_ens_* of include/em2g.h).

Each run of an ensemble must advance exactly as an ordinary FP32 context
of the same parameters does: after one step the particles are bitwise
equal (same arithmetic on the same fields), the fields differ only by the
order of the FP32 deposit atomics; over many steps the two stay within
FP32 round-off growth.  The graph replay and the direct launches do the
same work.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cfgs():
    from maccpic_b200.loader import HarrisConfig
    return [HarrisConfig(nx=64, ny=32, ppc=8, seed=1),
            HarrisConfig(nx=96, ny=48, ppc=4, seed=2, mass_ratio=49.0, psi0_over_b0di=0.13),
            HarrisConfig(nx=128, ny=64, ppc=6, seed=3, mass_ratio=100.0, isav=5)]


def _state(cfg):
    from maccpic_b200 import loader
    return loader.initial_fields(cfg), loader.sample_particles(cfg)


def _single(cfg, fld, parts):
    from maccpic_b200 import _lib
    from maccpic_b200.em2 import Em2Gpu
    n = parts[0].shape[1]
    g = Em2Gpu(cfg.run_params(np_max=[n, n], precision=_lib.FP32))
    g.set_fields(fld)
    for s, p in enumerate(parts):
        g.set_particles(s, p)
    return g


def _ensemble(cfgs, states):
    from maccpic_b200 import _lib
    from maccpic_b200.ensemble import Em2Ensemble
    runs = []
    for c, (fld, parts) in zip(cfgs, states):
        n = parts[0].shape[1]
        runs.append(c.run_params(np_max=[n, n], precision=_lib.FP32))
    e = Em2Ensemble(runs)
    for r, (fld, parts) in enumerate(states):
        e.set_fields(r, fld)
        for s, p in enumerate(parts):
            e.set_particles(r, s, p)
    return e


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def test_particle_roundtrip(gpu):
    cfgs = _cfgs()
    states = [_state(c) for c in cfgs]
    with _ensemble(cfgs, states) as e:
        for r, (_, parts) in enumerate(states):
            for s, p in enumerate(parts):
                q = e.get_particles(r, s)
                assert np.abs(q[:2] - p[:2]).max() < 1e-6
                np.testing.assert_allclose(q[2:], p[2:], rtol=1e-6, atol=1e-9)


def test_first_step_matches_single_runs(gpu):
    cfgs = _cfgs()
    states = [_state(c) for c in cfgs]
    with _ensemble(cfgs, states) as e:
        r_ens = e.step(1)
        for r, c in enumerate(cfgs):
            with _single(c, *states[r]) as g:
                r1 = g.step(1)
                assert r_ens["cg_iters"][r] == r1["cg_iters"]
                np.testing.assert_allclose(r_ens["ake"][r, :2], r1["ake"], rtol=1e-12)
                for s in range(2):
                    np.testing.assert_array_equal(e.get_particles(r, s), g.get_particles(s))
                fe, fg = e.get_fields(r), g.get_fields()
                for k in range(6):
                    assert rel(fe[k], fg[k]) < 1e-4, (r, k)


def test_many_steps_track_single_runs(gpu):
    """25 steps: every run crosses an isav step (filters and energies)."""
    cfgs = _cfgs()
    states = [_state(c) for c in cfgs]
    with _ensemble(cfgs, states) as e:
        out = None
        for _ in range(25):
            out = e.step(1)
        assert e.it == 25
        for r, c in enumerate(cfgs):
            with _single(c, *states[r]) as g:
                for _ in range(25):
                    r1 = g.step(1)
                np.testing.assert_allclose(out["ake"][r, :2], r1["ake"], rtol=1e-4)
                if 25 % c.isav == 0:
                    np.testing.assert_allclose(out["energies"][r], r1["energies"], rtol=1e-3,
                                               atol=1e-12)
                else:
                    assert np.isnan(out["energies"][r]).all()
                assert abs(int(out["cg_iters"][r]) - r1["cg_iters"]) <= 1
                fe, fg = e.get_fields(r), g.get_fields()
                for k in range(3, 6):
                    assert rel(fe[k], fg[k]) < 1e-3, (r, k)
                de, dg = e.diagnostics(r), g.diagnostics()
                np.testing.assert_allclose(de["flux"], dg["flux"], rtol=1e-3)


def test_graph_and_direct_launches_agree(gpu):
    cfgs = _cfgs()
    states = [_state(c) for c in cfgs]
    with _ensemble(cfgs, states) as a, _ensemble(cfgs, states) as b:
        b.set_graph(False)
        for _ in range(6):
            ra = a.step(1)
            rb = b.step(1)
        np.testing.assert_allclose(ra["ake"], rb["ake"], rtol=1e-4)
        ca, cb = a.counters(), b.counters()
        assert ca["graph_launches"] == 6 and cb["graph_launches"] == 0
        # one scan (3), push, kinetic energies, prescale, tick, 14 field stages
        assert ca["kernels_per_step"] == cb["kernels_per_step"] == 21
        assert ca["kernel_launches"] == 6 * 21
        for r in range(len(cfgs)):
            fa, fb = a.get_fields(r), b.get_fields(r)
            for k in range(3, 6):
                assert rel(fa[k], fb[k]) < 1e-4


def test_every_variant_runs(gpu):
    from maccpic_b200 import _lib
    from maccpic_b200.em2 import Em2Gpu
    cfgs = _cfgs()[:2]
    states = [_state(c) for c in cfgs]
    n = states[0][1][0].shape[1]
    with Em2Gpu(cfgs[0].run_params(np_max=[n, n], precision=_lib.FP32)) as g:
        nvar = g.num_variants()
    assert nvar >= 8
    with _ensemble(cfgs, states) as ref:
        ref.step(1)
        want = [[ref.get_particles(r, s) for s in range(2)] for r in range(2)]
        for v in range(1, nvar):
            with _ensemble(cfgs, states) as e:
                e.set_variant(v)
                e.step(1)
                for r in range(2):
                    for s in range(2):
                        np.testing.assert_array_equal(e.get_particles(r, s), want[r][s])


def test_current_filter_in_an_ensemble(gpu):
    import dataclasses
    cfgs = [dataclasses.replace(c, smooth_current=1) for c in _cfgs()[:2]]
    states = [_state(c) for c in cfgs]
    with _ensemble(cfgs, states) as e:
        e.step(3)
        assert e.counters()["kernels_per_step"] == 23
        for r, c in enumerate(cfgs):
            with _single(c, *states[r]) as g:
                g.step(3)
                fe, fg = e.get_fields(r), g.get_fields()
                for k in range(6):
                    assert rel(fe[k], fg[k]) < 1e-4, (r, k)


def test_errors(gpu):
    from maccpic_b200 import _lib
    from maccpic_b200._lib import Em2gError
    cfgs = _cfgs()[:2]
    states = [_state(c) for c in cfgs]
    e = _ensemble(cfgs, states)
    with e:
        with pytest.raises(Em2gError) as ei:
            e.set_particles(0, 0, states[0][1][0][:, :10])
        assert ei.value.status == _lib.ERR_RANGE
        bad = states[0][1][0].copy()
        bad[0, 3] = cfgs[0].nx + 1.0
        with pytest.raises(Em2gError) as ei:
            e.set_particles(0, 0, bad)
        assert ei.value.status == _lib.ERR_RANGE
        with pytest.raises(IndexError):
            e.get_fields(5)
    from maccpic_b200.ensemble import Em2Ensemble
    n = states[0][1][0].shape[1]
    with Em2Ensemble([cfgs[0].run_params(np_max=[n, n], precision=_lib.FP32)]) as f:
        with pytest.raises(Em2gError) as ei:
            f.step(1)
        assert ei.value.status == _lib.ERR_INVALID


def test_sort_interval_tracks_single_runs(gpu):
    """With a sort interval the ensemble pushes in place between regroupings,
    as single contexts do: after the first step (in place) the particles are
    bitwise those of single runs at the same interval, and over 7 steps at
    interval 3 (two regroupings) the runs track them."""
    cfgs = _cfgs()
    states = [_state(c) for c in cfgs]
    singles = [_single(c, *states[r]) for r, c in enumerate(cfgs)]
    try:
        with _ensemble(cfgs, states) as e:
            e.set_sort_interval(3)
            for g in singles:
                g.set_sort_interval(3)
            e.step(1)
            assert e.counters()["kernels_per_step"] == 18  # no scan in place
            for r, g in enumerate(singles):
                g.step(1)
                for s in range(2):
                    np.testing.assert_array_equal(e.get_particles(r, s), g.get_particles(s))
            out = None
            for _ in range(6):
                out = e.step(1)
            assert e.it == 7 and e.counters()["graph_launches"] == 7
            for r, g in enumerate(singles):
                r1 = None
                for _ in range(6):
                    r1 = g.step(1)
                np.testing.assert_allclose(out["ake"][r, :2], r1["ake"], rtol=1e-4)
                fe, fg = e.get_fields(r), g.get_fields()
                for k in range(3, 6):
                    assert rel(fe[k], fg[k]) < 1e-3, (r, k)
                for s in range(2):
                    pe, pg = e.get_particles(r, s), g.get_particles(s)
                    assert np.abs(pe[:2] - pg[:2]).max() < 1e-3
    finally:
        for g in singles:
            g.close()


def test_sort_interval_rules(gpu):
    """k * c * dt < dx, dy in every run; runs created together share one
    interval."""
    import dataclasses
    from maccpic_b200 import _lib
    from maccpic_b200._lib import Em2gError
    from maccpic_b200.ensemble import Em2Ensemble
    cfgs = _cfgs()[:2]
    states = [_state(c) for c in cfgs]
    with _ensemble(cfgs, states) as e:
        kmax = e.max_sort_interval()
        assert kmax > 1
        with pytest.raises(Em2gError) as ei:
            e.set_sort_interval(kmax + 1)
        assert ei.value.status == _lib.ERR_INVALID
        with pytest.raises(Em2gError):
            e.set_sort_interval(-1)
        e.set_sort_interval(kmax)
        e.step(kmax + 1)
        e.set_sort_interval(0)
        e.step(1)
    n = [s[1][0].shape[1] for s in states]
    runs = [c.run_params(np_max=[k, k], precision=_lib.FP32) for c, k in zip(cfgs, n)]
    runs[0] = dataclasses.replace(runs[0], sort_interval=2)
    with pytest.raises(Em2gError) as ei:
        Em2Ensemble(runs)
    assert ei.value.status == _lib.ERR_INVALID
    runs[1] = dataclasses.replace(runs[1], sort_interval=2)
    with Em2Ensemble(runs) as f:
        assert all(r.sort_interval == 2 for r in f.runs)


def test_outputs_into_caller_buffers(gpu):
    """The ensemble's getters fill a caller's buffer (pinned memory here) with
    what they would return, as a context's do."""
    import torch
    cfgs = _cfgs()[:2]
    states = [_state(c) for c in cfgs]
    with _ensemble(cfgs, states) as e:
        e.step(2)
        for r in range(2):
            want = e.get_fields(r)
            out = torch.empty(want.shape, dtype=torch.float64).pin_memory().numpy()
            assert e.get_fields(r, out=out) is out
            np.testing.assert_array_equal(out, want)
            for s in range(2):
                want = e.get_particles(r, s)
                out = torch.empty(want.shape, dtype=torch.float64).pin_memory().numpy()
                e.get_particles(r, s, out=out)
                np.testing.assert_array_equal(out, want)
        with pytest.raises(ValueError):
            e.get_particles(0, 0, out=np.empty((5, 3)))


def test_runs_against_the_oracle(gpu, oracle_lib):
    """Every run of an ensemble -- mass ratios 25, 49 and 100, uneven grids --
    against the FP64 oracle stepping the same state, at the mixed path's
    tolerances (those of test_gpu_fp32): kinetic energies to 1e-5 relative
    every step, total field energy to 1e-4 at the isav steps, E and B to
    1e-2 of their largest value and positions to 1e-3 cells after 40
    steps; the FP64 reconnected flux and energies the ensemble reports for a
    run equal a host computation from its downloaded fields."""
    cfgs = _cfgs()
    states = [_state(c) for c in cfgs]
    oracles = []
    for c, (fld, parts) in zip(cfgs, states):
        rp = c.run_params()
        op = oracle_lib.Params(nx=c.nx, ny=c.ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, qm=rp.qm, q=rp.q,
                               dn=rp.dn, am=rp.am, isav=rp.isav)
        oracles.append(oracle_lib.State(op, fld, parts))
    with _ensemble(cfgs, states) as e:
        for k in range(1, 41):
            r = e.step(1)
            for i, (c, st) in enumerate(zip(cfgs, oracles)):
                ref = st.step()
                np.testing.assert_allclose(r["ake"][i, :2], ref["ake"], rtol=1e-5)
                assert r["cg_iters"][i] >= 1
                if k % c.isav == 0:
                    tot, tot_ref = r["energies"][i].sum(), ref["energies"].sum()
                    assert abs(tot - tot_ref) / tot_ref < 1e-4, (i, k, tot, tot_ref)
        for i, (c, st) in enumerate(zip(cfgs, oracles)):
            got = e.get_fields(i)
            for f in range(6):
                scale = np.abs(st.fld[f]).max()
                assert np.abs(got[f] - st.fld[f]).max() / scale < 1e-2, (i, f)
            for s in range(2):
                q = e.get_particles(i, s)
                for ax, n in ((0, c.nx), (1, c.ny)):
                    d = np.abs(q[ax] - st.parts[s][ax])
                    assert np.minimum(d, n - d).max() < 1e-3, (i, s, ax)
            d = e.diagnostics(i)
            a = got[:6, 1:c.ny + 1, 1:c.nx + 1]
            e6 = 0.5 * (a * a).sum(axis=(1, 2)) / (c.nx * c.ny)
            np.testing.assert_allclose(d["energies"], e6, rtol=1e-12)
            by = got[4]
            for sheet, row in enumerate((c.ny // 4, c.ny // 4 + c.ny // 2)):
                b = 0.5 * (by[row, 1:c.nx + 1] + by[row + 1, 1:c.nx + 1])
                psi = -np.cumsum(b) * c.dx
                np.testing.assert_allclose(d["flux"][sheet], psi.max() - psi.min(), rtol=1e-11)


@pytest.mark.parametrize("graph,interval,smooth", [(True, 1, 0), (False, 1, 0), (True, 3, 0),
                                                   (True, 1, 1)],
                         ids=["graph", "direct", "in-place", "current-filter"])
def test_fused_step_matches_staged_launches(gpu, graph, interval, smooth):
    """The step as one persistent, cooperative launch (em2g_ens_set_fused)
    against the stage-by-stage launches: after one step the particles are
    bitwise equal (the same arithmetic on the same fields) and the kinetic
    energies equal to their summation order; over the next steps, the FP32
    deposit atomics adding in another order, fields, energies and kinetic
    energies stay within FP32 round-off growth.  The runs' isav of 20, 20 and
    5 exercise the E/B filter and the energies inside the launch."""
    import dataclasses
    cfgs = [dataclasses.replace(c, smooth_current=smooth) for c in _cfgs()]
    states = [_state(c) for c in cfgs]
    with _ensemble(cfgs, states) as a, _ensemble(cfgs, states) as b:
        b.set_fused(True)
        b.set_graph(graph)
        a.set_sort_interval(interval)
        b.set_sort_interval(interval)
        ra, rb = a.step(1), b.step(1)
        np.testing.assert_allclose(rb["ake"], ra["ake"], rtol=1e-12)
        for r in range(len(cfgs)):
            for s in range(2):
                np.testing.assert_array_equal(b.get_particles(r, s), a.get_particles(r, s))
        assert b.counters()["kernels_per_step"] == 1
        for _ in range(9):
            ra, rb = a.step(1), b.step(1)
        np.testing.assert_allclose(rb["ake"], ra["ake"], rtol=1e-4)
        assert (rb["cg_iters"] >= 1).all()
        for r, c in enumerate(cfgs):
            fa, fb = a.get_fields(r), b.get_fields(r)
            for k in range(6):
                assert rel(fb[k], fa[k]) < 1e-3, (r, k)
            if 10 % c.isav == 0:
                np.testing.assert_allclose(rb["energies"][r], ra["energies"][r], rtol=1e-4)
        if graph:
            assert b.counters()["graph_launches"] == 10
