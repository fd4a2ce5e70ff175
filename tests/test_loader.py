"""The seeded double-Harris loader (maccpic_b200/loader.py, host sampler) on
the CPU: the initial B has zero discrete divergence on em2's staggered grid;
the sampled density follows n_b (1 + csden sech^2) in y and is uniform in
x; the sheet particles drift along z so that the current n0 (V_i - V_e)
equals the B0/L of the Harris profile's curl, with the signs each sheet
needs; temperatures satisfy the pressure balance B0^2/2 = n0 (Te + Ti); every
particle is inside the box with |v| < 1 and gamma = 1/sqrt(1 - v^2); and the
same seed gives the same particles.
"""
import numpy as np


def _cfg(**kw):
    from maccpic_b200 import loader
    base = dict(nx=64, ny=128, ppc=64, seed=3)
    base.update(kw)
    return loader.HarrisConfig(**base)


def test_initial_b_is_divergence_free_on_the_staggered_grid():
    from maccpic_b200 import loader
    from maccpic_b200._lib import FIELD_ID
    cfg = _cfg(guide_over_b0=0.3)
    f = loader.initial_fields(cfg)
    bx, by = f[FIELD_ID["bx"]], f[FIELD_ID["by"]]
    # Bx(iy, ix) at (ix-1/2, iy-1), By(iy, ix) at (ix-1, iy-1/2): div B at the
    # integer node (ix-1, iy-1) is Bx(iy, ix) - Bx(iy, ix-1) + By(iy, ix) - By(iy-1, ix)
    div = (bx[1:, 1:] - bx[1:, :-1]) + (by[1:, 1:] - by[:-1, 1:])
    assert np.abs(div).max() < 1e-13 * max(np.abs(bx).max(), 1.0)
    assert np.all(f[FIELD_ID["bz"]] == cfg.guide_over_b0 * cfg.b0)
    for k in ("ex", "ey", "ez", "rho", "jxm", "jzp"):
        assert not f[FIELD_ID[k]].any()
    # Bx = B0 [tanh((y-y1)/L) - tanh((y-y2)/L) - 1]: +B0 between the sheets,
    # -B0 outside them, reversing across each
    col = bx[:, cfg.nx // 2 + 1]
    assert col[cfg.ny // 2 + 1] > 0.9 * cfg.b0 and col[1] < -0.9 * cfg.b0


def test_density_drifts_and_temperatures():
    from maccpic_b200 import loader
    cfg = _cfg()
    e, i = loader.sample_particles(cfg)
    n = cfg.nx * cfg.ny * cfg.ppc
    assert e.shape == (6, n) and i.shape == (6, n)
    np.testing.assert_array_equal(e[:2], i[:2])  # quasi-neutral: shared positions
    x, y = e[0], e[1]
    assert x.min() >= 0 and x.max() < cfg.nx and y.min() >= 0 and y.max() < cfg.ny
    # density in y against n_b (1 + csden sech^2) over both sheets
    lc = cfg.L / cfg.dx
    edges = np.arange(cfg.ny + 1, dtype=float)
    cnt, _ = np.histogram(y, edges)
    yc = edges[:-1] + 0.5
    prof = 1.0 + cfg.csden * (np.cosh((yc - cfg.ny / 4) / lc) ** -2
                              + np.cosh((yc - 3 * cfg.ny / 4) / lc) ** -2)
    want = n * prof / prof.sum()
    assert np.abs(cnt - want).max() < 6 * np.sqrt(want.max())
    # uniform in x
    cx, _ = np.histogram(x, np.arange(cfg.nx + 1, dtype=float))
    assert np.abs(cx - n / cfg.nx).max() < 6 * np.sqrt(n / cfg.nx)
    # pressure balance
    te, ti = cfg.temperatures()
    assert abs(cfg.b0 ** 2 / 2 - cfg.csden * (te + ti)) < 1e-14
    assert abs(ti / te - cfg.ti_over_te) < 1e-12
    # relativistic consistency
    for p in (e, i):
        v2 = p[2] ** 2 + p[3] ** 2 + p[4] ** 2
        assert v2.max() < 1.0
        np.testing.assert_allclose(p[5], 1.0 / np.sqrt(1.0 - v2), rtol=1e-12)


def test_sheet_current_matches_the_curl_of_b():
    """n0 (V_i - V_e) = B0/L at each sheet centre, with opposite signs on
    the two sheets, as -dBx/dy of the Harris profile requires."""
    from maccpic_b200 import loader
    cfg = _cfg(ppc=128)
    e, i = loader.sample_particles(cfg)
    lc = cfg.L / cfg.dx
    # the drift of the particles near each sheet centre (|y - c| < L/4),
    # where the sheet population dominates the background 1 : csden
    out = []
    for c in (cfg.ny / 4, 3 * cfg.ny / 4):
        sel = np.abs(e[1] - c) < 0.25 * lc
        frac_sheet = cfg.csden / (1.0 + cfg.csden)  # at the centre, sech^2 ~ 1
        # per-particle momentum-weighted drift: mean of gamma vz
        ue = (e[5] * e[4])[sel].mean() / frac_sheet
        ui = (i[5] * i[4])[sel].mean() / frac_sheet
        out.append((ue, ui))
    vdiff = cfg.b0 / (cfg.L * cfg.csden)
    (ue1, ui1), (ue2, ui2) = out
    # opposite drifts on the two sheets, ions against electrons
    assert np.sign(ui1) == -np.sign(ue1) and np.sign(ui2) == -np.sign(ue2)
    assert np.sign(ui1) == -np.sign(ui2)
    # magnitudes: the drift difference gives the sheet current within the
    # sampling noise and the background's share (a few per cent)
    for ue, ui in out:
        assert abs(abs(ui - ue) / vdiff - 1.0) < 0.08
    # the sign of sheet 1's current, -dBx/dy there (Bx rises through y1)
    from maccpic_b200._lib import FIELD_ID
    f = loader.initial_fields(cfg)
    bx = f[FIELD_ID["bx"]][:, cfg.nx // 2 + 1]
    iy1 = int(cfg.ny / 4) + 1
    curl_z = -(bx[iy1 + 1] - bx[iy1 - 1]) / (2 * cfg.dx)
    jz1 = ui1 - ue1  # charge +1 ions, -1 electrons
    assert np.sign(jz1) == np.sign(curl_z)


def test_same_seed_same_particles_other_seed_others():
    from maccpic_b200 import loader
    a = loader.sample_particles(_cfg(nx=16, ny=16, ppc=4, seed=9))
    b = loader.sample_particles(_cfg(nx=16, ny=16, ppc=4, seed=9))
    c = loader.sample_particles(_cfg(nx=16, ny=16, ppc=4, seed=10))
    for p, q in zip(a, b):
        np.testing.assert_array_equal(p, q)
    assert not np.array_equal(a[0], c[0])
