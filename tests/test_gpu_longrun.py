"""A whole run against the oracle, compared within the seed-to-seed spread.

The double-Harris workload at 256x128 cells, 16 particles per cell per
species, runs its full 2000 steps on the GPU (FP64, em2's arithmetic) and on
the oracle from the same seeded state; five more seeds on the GPU give the
spread that particle noise alone produces.  At every diagnostic time (every
20 steps) the GPU-oracle difference of the total energy, the reconnected
flux of both sheets and the reconnection rate (the flux's time derivative)
must lie inside that spread; so must the mixed FP32 path's.  Over the first
300 steps, before the two FP64 runs' different summation orders have grown
into visibly different particle trajectories, the FP64 difference must stay
below 1e-3 of the spread.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS, EVERY = 2000, 20
TIGHT = 300 // EVERY  # diagnostic times held to 1e-3 of the spread
SEEDS = 6


def flux(fld, nx, ny, dx, j):
    """max - min of psi = -integral of By dx along the centre row of the
    sheet between rows j and j+1 (By of the two rows averaged)."""
    by = fld[4]
    b = 0.5 * (by[j, 1:nx + 1] + by[j + 1, 1:nx + 1])
    psi = -np.cumsum(b) * dx
    return psi.max() - psi.min()


def quantities(fld, ake, cfg):
    nx, ny = cfg.nx, cfg.ny
    return (field_energy(fld, nx, ny) + float(np.sum(ake)),
            flux(fld, nx, ny, cfg.dx, ny // 4), flux(fld, nx, ny, cfg.dx, ny // 4 + ny // 2))


def field_energy(fld, nx, ny):
    a = fld[:6, 1:ny + 1, 1:nx + 1]
    return 0.5 * float(np.sum(a * a)) / (nx * ny)


def series_gpu(cfg, precision):
    from maccpic_b200 import loader
    from maccpic_b200.em2 import Em2Gpu
    fld, parts = loader.initial_state(cfg)
    out = []
    with Em2Gpu(cfg.run_params(precision=precision)) as g:
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        for k in range(STEPS // EVERY):
            r = g.step(EVERY)
            out.append(quantities(g.get_fields(), r["ake"], cfg))
    return np.array(out)


def series_oracle(cfg, oracle):
    from maccpic_b200 import loader
    fld, parts = loader.initial_state(cfg)
    rp = cfg.run_params()
    op = oracle.Params(nx=cfg.nx, ny=cfg.ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, qm=rp.qm, q=rp.q,
                       dn=rp.dn, am=rp.am, isav=rp.isav)
    st = oracle.State(op, fld, parts)
    out = []
    for k in range(STEPS // EVERY):
        for _ in range(EVERY):
            r = st.step(nthreads=os.cpu_count() or 1)
        out.append(quantities(st.fld, r["ake"], cfg))
    return np.array(out)


def test_run_within_seed_spread(gpu, oracle_lib):
    import dataclasses
    from maccpic_b200 import _lib, loader
    base = loader.PRESETS["harris_256x128_ppc16"]
    assert base.steps == STEPS
    gpu64 = [series_gpu(dataclasses.replace(base, seed=s), _lib.FP64) for s in range(SEEDS)]
    ref = series_oracle(base, oracle_lib)
    f32 = series_gpu(base, _lib.FP32)
    seeds = np.array(gpu64)                          # (seed, time, quantity)
    dt = EVERY * base.dt
    rate = np.diff(seeds[:, :, 1:], axis=1) / dt     # reconnection rates d flux / dt
    spread = seeds.max(0) - seeds.min(0)
    spread_rate = rate.max(0) - rate.min(0)
    assert (spread[1:] > 0).all()
    for name, s in (("gpu fp64", gpu64[0]), ("gpu fp32", f32)):
        d = np.abs(s - ref)
        print(name, "max |diff| / spread per quantity:",
              (d / (spread + 1e-300)).max(0), "final:", (d[-1] / spread[-1]))
        assert (d <= spread + 1e-9 * np.abs(ref)).all(), (name, np.argwhere(d > spread))
        r_s = np.diff(s[:, 1:], axis=0) / dt
        r_ref = np.diff(ref[:, 1:], axis=0) / dt
        dr = np.abs(r_s - r_ref)
        assert (dr <= spread_rate + 1e-9).all(), (name, np.argwhere(dr > spread_rate))
    # the FP64 path stays far inside the spread while the summation orders
    # have not yet grown into different trajectories
    d = np.abs(gpu64[0] - ref)[:TIGHT]
    assert (d <= 1e-3 * spread[:TIGHT] + 1e-9 * np.abs(ref[:TIGHT])).all()
