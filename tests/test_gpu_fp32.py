"""The mixed-precision path (FP32 particles, gather, deposit, Yee; FP64
reductions) against the FP64 oracle.  FP32 arithmetic cannot be bitwise; the
bounds below are the ones the mixed path is held to:
  * positions round-trip through the cell-relative FP32 layout to < 2e-7
    cells, velocities to < 1e-6 relative;
  * after 50 steps of the double-Harris workload the field energy differs
    from the FP64 oracle's by < 1e-4 relative and E, B by < 1e-2 of their
    max |value| (the mixed path is meant to stay within 1e-3 on the field energy).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def harris(nx=128, ny=64, ppc=16, seed=2):
    import oracle
    from maccpic_b200 import loader, _lib
    cfg = loader.HarrisConfig(nx=nx, ny=ny, ppc=ppc, seed=seed)
    fld, parts = loader.initial_state(cfg)
    rp = cfg.run_params(precision=_lib.FP32)
    op = oracle.Params(nx=nx, ny=ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, qm=rp.qm, q=rp.q,
                       dn=rp.dn, am=rp.am, isav=rp.isav)
    return op, rp, fld, parts


def test_fp32_particle_roundtrip(gpu):
    from maccpic_b200.em2 import Em2Gpu
    op, rp, fld, parts = harris(nx=64, ny=32, ppc=8)
    with Em2Gpu(rp) as g:
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        for s, p in enumerate(parts):
            q = g.get_particles(s)
            assert np.abs(q[:2] - p[:2]).max() < 2e-7 * 4  # cells (offsets < 1, FP32)
            np.testing.assert_allclose(q[2:5], p[2:5], rtol=1e-6, atol=1e-9)
            np.testing.assert_allclose(q[5], p[5], rtol=1e-6)


def test_fp32_fields_roundtrip(gpu):
    from maccpic_b200.em2 import Em2Gpu
    op, rp, fld, parts = harris(nx=64, ny=32, ppc=8)
    with Em2Gpu(rp) as g:
        g.set_fields(fld)
        np.testing.assert_allclose(g.get_fields(), fld.astype(np.float32).astype(np.float64))


def test_outputs_into_caller_buffers(gpu):
    """get_fields / get_particles fill a caller's buffer (pinned memory here)
    with what they would return; a buffer of the wrong shape is refused."""
    import torch
    from maccpic_b200.em2 import Em2Gpu
    op, rp, fld, parts = harris(nx=64, ny=32, ppc=8)
    with Em2Gpu(rp) as g:
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        out_f = torch.empty(fld.shape, dtype=torch.float64).pin_memory().numpy()
        assert g.get_fields(out=out_f) is out_f
        np.testing.assert_array_equal(out_f, g.get_fields())
        for s, p in enumerate(parts):
            out_p = torch.empty(p.shape, dtype=torch.float64).pin_memory().numpy()
            g.get_particles(s, out=out_p)
            np.testing.assert_array_equal(out_p, g.get_particles(s))
        with pytest.raises(ValueError):
            g.get_particles(0, out=np.empty((6, parts[0].shape[1] - 1)))
        with pytest.raises(ValueError):
            g.get_fields(out=np.empty(fld.shape, dtype=np.float32))


def test_fp32_step_against_fp64_oracle(gpu, oracle_lib):
    from maccpic_b200.em2 import Em2Gpu
    op, rp, fld, parts = harris()
    st = oracle_lib.State(op, fld, parts)
    e_ref = e_got = None
    with Em2Gpu(rp) as g:
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        for k in range(1, 41):
            r_ref = st.step()
            r = g.step(1)
            np.testing.assert_allclose(r["ake"], r_ref["ake"], rtol=1e-5)
            if k % rp.isav == 0:
                e_ref, e_got = r_ref["energies"], r["energies"]
                tot_ref, tot = e_ref.sum(), e_got.sum()
                assert abs(tot - tot_ref) / tot_ref < 1e-4, (k, tot, tot_ref)
        got = g.get_fields()
        for k in range(6):
            scale = np.abs(st.fld[k]).max()
            err = np.abs(got[k] - st.fld[k]).max() / scale
            print(oracle_lib.FIELD_NAMES[k], err)
            assert err < 1e-2, (oracle_lib.FIELD_NAMES[k], err)
        for s in range(2):
            q = g.get_particles(s)
            dx = np.abs(q[0] - st.parts[s][0])
            dx = np.minimum(dx, rp.nx - dx)  # periodic
            assert dx.max() < 1e-3
    assert e_ref is not None


def test_fp32_rejects_split_move_curnt(gpu):
    from maccpic_b200.em2 import Em2Gpu
    from maccpic_b200._lib import Em2gError, ERR_INVALID
    op, rp, fld, parts = harris(nx=32, ny=16, ppc=4)
    with Em2Gpu(rp) as g:
        with pytest.raises(Em2gError) as ei:
            g.move()
        assert ei.value.status == ERR_INVALID


def test_fp32_variants_agree(gpu):
    """All FP32 push variants give the same fields to FP32 rounding."""
    from maccpic_b200.em2 import Em2Gpu
    op, rp, fld, parts = harris(nx=128, ny=32, ppc=8)
    outs = []
    with Em2Gpu(rp) as probe:
        n = probe.num_variants()
    for v in range(n):
        with Em2Gpu(rp) as g:
            g.set_variant(v)
            g.set_fields(fld)
            for s, p in enumerate(parts):
                g.set_particles(s, p)
            for _ in range(5):
                g.step(1)
            outs.append(g.get_fields())
    for v in range(1, n):
        for k in range(6):
            err = np.abs(outs[v][k] - outs[0][k]).max() / np.abs(outs[0][k]).max()
            assert err < 1e-4, (v, k, err)


def _relativistic(nx=48, ny=32, n=6000, seed=4):
    """Random fields and particles up to gamma ~ 5 (|v| up to 0.98 c): the
    largest per-step drift the interval bound has to hold."""
    from maccpic_b200 import _lib
    from maccpic_b200.em2 import RunParams
    rng = np.random.default_rng(seed)
    fld = np.zeros((13, ny + 3, nx + 3))
    f = rng.normal(scale=0.05, size=(6, ny, nx))
    iy = (np.arange(ny + 3) - 1) % ny
    ix = (np.arange(nx + 3) - 1) % nx
    fld[:6] = f[:, iy][:, :, ix]
    parts = []
    for s in range(2):
        u = rng.normal(size=(3, n)) * (2.5 if s == 0 else 0.3)
        g = np.sqrt(1 + (u * u).sum(0))
        parts.append(np.vstack([rng.random(n) * nx, rng.random(n) * ny, u / g, g]))
    rp = RunParams(nx=nx, ny=ny, dx=0.5, dy=0.5, dt=0.05, qm=[-1.0, 1 / 25.0],
                   q=[-0.01, 0.01], dn=[1.0, 1.0], am=[0.01, 0.25], np_max=[n, n],
                   precision=_lib.FP32)
    return rp, fld, parts


@pytest.mark.parametrize("k", [2, 9])
def test_sort_interval_matches_regrouping_every_step(gpu, k):
    """In-place pushes between regroupings give the same run (to FP32
    round-off) as regrouping every step, at the largest interval the drift
    bound allows (9 at c dt / dx = 0.1) with particles near c."""
    from maccpic_b200.em2 import Em2Gpu
    rp, fld, parts = _relativistic()
    with Em2Gpu(rp) as a, Em2Gpu(rp) as b:
        assert b.max_sort_interval() == 9
        for g in (a, b):
            g.set_fields(fld)
            for s, p in enumerate(parts):
                g.set_particles(s, p)
        b.set_sort_interval(k)
        for _ in range(3 * k + 1):
            ra, rb = a.step(1), b.step(1)
            np.testing.assert_allclose(rb["ake"], ra["ake"], rtol=1e-5)
        for s in range(2):
            pa, pb = a.get_particles(s), b.get_particles(s)
            d = np.abs(pa[:2] - pb[:2])
            d = np.minimum(d, np.array([[rp.nx], [rp.ny]]) - d)
            assert d.max() < 1e-4
            np.testing.assert_allclose(pb[2:], pa[2:], rtol=1e-3, atol=1e-5)
        fa, fb = a.get_fields(), b.get_fields()
        for c in range(6):
            assert np.abs(fa[c] - fb[c]).max() < 1e-4 * np.abs(fa[c]).max() + 1e-7


def test_sort_interval_rejected_beyond_the_drift_bound(gpu):
    from maccpic_b200 import _lib
    from maccpic_b200._lib import Em2gError
    from maccpic_b200.em2 import Em2Gpu
    rp, fld, parts = _relativistic()
    with Em2Gpu(rp) as g:
        with pytest.raises(Em2gError) as ei:
            g.set_sort_interval(10)
        assert ei.value.status == _lib.ERR_INVALID
        g.set_sort_interval(9)


def test_offsets_that_round_up_to_the_next_cell(gpu, oracle_lib):
    """Positions a hair below a cell edge, whose FP32 offset rounds to
    exactly 1, belong to the next cell in the FP32 layout: the upload groups
    them there, and in-place pushes keep each offset inside the cell they
    counted for the next grouping.  Every particle is placed (a push that
    found no place for one would fail the step), and the run tracks the
    oracle to the mixed path's bounds."""
    import oracle
    from maccpic_b200 import _lib
    from maccpic_b200.em2 import Em2Gpu, RunParams
    nx, ny, n = 32, 16, 4000
    kw = dict(nx=nx, ny=ny, dx=0.5, dy=0.5, dt=0.05, qm=[-1.0, 1 / 25.0], q=[-0.02, 0.02],
              dn=[1.0, 1.0], am=[0.02, 0.5], isav=4)
    rng = np.random.default_rng(5)
    x, y = rng.random(n) * nx, rng.random(n) * ny
    k = np.arange(600)
    x[:600] = (k % nx) + 1 - 1e-12  # includes nx - 1e-12, which wraps to cell 0
    y[300:900] = (k % ny) + 1 - 1e-12
    parts = []
    for s in range(2):  # both species on the same positions: no net charge
        u = rng.normal(scale=0.2 if s == 0 else 0.04, size=(3, n))
        g = np.sqrt(1 + (u * u).sum(0))
        parts.append(np.vstack([x, y, u / g, g]))
    fld = np.zeros((13, ny + 3, nx + 3))
    st = oracle_lib.State(oracle.Params(**kw), fld, parts)
    rp = RunParams(np_max=[n, n], precision=_lib.FP32, **kw)
    with Em2Gpu(rp) as g:
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        q0 = g.get_particles(0)
        d = np.abs(q0[:2] - parts[0][:2])
        d = np.minimum(d, np.array([[nx], [ny]]) - d)
        assert d.max() < 1e-6
        g.set_sort_interval(g.max_sort_interval())
        for _ in range(12):
            st.step()
            g.step(1)
        for s in range(2):
            p = g.get_particles(s)
            d = p[:2] - st.parts[s][:2]
            d -= np.array([[nx], [ny]]) * np.round(d / np.array([[nx], [ny]]))
            assert np.abs(d).max() < 1e-3
        got = g.get_fields()
        for f in range(6):
            scale = max(np.abs(st.fld[f]).max(), 1e-30)
            assert np.abs(got[f] - st.fld[f]).max() / scale < 1e-2, f


def test_autotuner_keeps_the_fastest_variant_and_interval(gpu):
    """The autotuner times the fastest few variants at every admissible sort
    interval and leaves the context on the best pair it timed."""
    from maccpic_b200 import autotune
    from maccpic_b200.em2 import Em2Gpu
    op, rp, fld, parts = harris(nx=128, ny=64, ppc=16)
    with Em2Gpu(rp) as g:
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        r = autotune.autotune(g, particles=parts[0].shape[1], cache=None, use_cache=False)
        assert len(r["times_ms"]) == g.num_variants()
        assert str(r["variant"]) in r["candidates"]
        kmax = g.max_sort_interval()
        for v, ms in r["candidates"].items():
            assert set(ms) == {str(k) for k in (1, 2, 3, 4, 6, kmax) if k <= kmax}
        best = min(t for ms in r["candidates"].values() for t in ms.values())
        assert r["candidates"][str(r["variant"])][str(r["sort_interval"])] == best
        assert g.variant()[0] == r["variant"] and g.p.sort_interval == r["sort_interval"]
        g.step(2)
