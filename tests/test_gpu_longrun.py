"""A whole run against the oracle, compared within the seed-to-seed spread.

The double-Harris workload at 256x128 cells, 16 particles per cell per
species, runs 300 steps on the GPU (FP64, em2's arithmetic) and on the oracle
from the same seeded state; four more seeds on the GPU give the spread that
particle noise alone produces.  At every diagnostic time the GPU-oracle
difference of the total energy, the reconnected flux and the reconnection
rate (its time derivative) must lie inside that spread; so must the mixed
FP32 path's.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS, EVERY = 300, 20


def flux(fld, nx, ny, dx):
    """max - min of psi = -integral of By dx along the centre row of the
    sheet at ny/4 (By of rows ny/4 and ny/4+1 averaged)."""
    by = fld[4]
    j = ny // 4
    b = 0.5 * (by[j, 1:nx + 1] + by[j + 1, 1:nx + 1])
    psi = -np.cumsum(b) * dx
    return psi.max() - psi.min()


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
            f = g.get_fields()
            out.append((field_energy(f, cfg.nx, cfg.ny) + float(np.sum(r["ake"])),
                        flux(f, cfg.nx, cfg.ny, cfg.dx)))
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
        out.append((field_energy(st.fld, cfg.nx, cfg.ny) + float(np.sum(r["ake"])),
                    flux(st.fld, cfg.nx, cfg.ny, cfg.dx)))
    return np.array(out)


def test_run_within_seed_spread(gpu, oracle_lib):
    import dataclasses
    from maccpic_b200 import _lib, loader
    base = loader.PRESETS["harris_256x128_ppc16"]
    gpu64 = [series_gpu(dataclasses.replace(base, seed=s), _lib.FP64) for s in range(5)]
    ref = series_oracle(base, oracle_lib)
    f32 = series_gpu(base, _lib.FP32)
    seeds = np.array(gpu64)                          # (seed, time, quantity)
    dt = EVERY * base.dt
    rate = np.diff(seeds[:, :, 1], axis=1) / dt      # reconnection rate d flux / dt
    spread = seeds.max(0) - seeds.min(0)
    spread_rate = rate.max(0) - rate.min(0)
    assert (spread[1:] > 0).all()
    for name, s in (("gpu fp64", gpu64[0]), ("gpu fp32", f32)):
        for q in range(2):
            assert (np.abs(s[:, q] - ref[:, q]) <= spread[:, q] + 1e-9 * np.abs(ref[:, q])).all(), \
                (name, q, s[:, q] - ref[:, q], spread[:, q])
        r_s = np.diff(s[:, 1]) / dt
        r_ref = np.diff(ref[:, 1]) / dt
        assert (np.abs(r_s - r_ref) <= spread_rate + 1e-9).all(), (name, r_s - r_ref, spread_rate)
    # the FP64 path stays far inside the spread: summation order only
    assert (np.abs(gpu64[0] - ref) <= 1e-3 * spread + 1e-9 * np.abs(ref)).all()
