"""The CPU oracle: pinned to the reference's published numbers, frozen by
golden vectors, and checked on known-answer cases (no GPU needed)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def em2_start(oracle_lib):
    """em2's own start-up, restated, at the test setup of
    pic/RECONNECTION_MODEL.md:454-460 (nx = 64, nproc = 2)."""
    setup = oracle_lib.Em2Setup(nx=64, nproc=2)
    params, st, maxnp = oracle_lib.em2_startup(setup)
    return setup, params, st, maxnp


def test_em2_initial_state_known_answers(oracle_lib, em2_start):
    gold = json.load(open(os.path.join(HERE, "golden", "em2_initial_state.json")))
    setup, params, st, maxnp = em2_start
    nx, ny, npcel = setup.nx, setup.ny, setup.npcel
    st = st.copy()
    # density from the loaded rows (both species are at the same positions)
    y = st.parts[0][1]
    centre = np.count_nonzero(np.abs(y - ny / 4) < 0.25) / (nx * npcel * 0.5)
    band = (y >= 40) & (y < 80)
    background = np.count_nonzero(band) / (nx * npcel * 40.0)
    assert round(centre, 1) == gold["density_sheet_centre"]
    assert round(background, 1) == gold["density_background"]
    # step 0: move, then mean vz of the sheet-1 slots (pic/creator.f90:204-226)
    st.move()
    nph = maxnp // 2
    npback = nx * ny * npcel // setup.nproc
    i = np.arange(1, maxnp + 1)
    bg = ((i <= npback // 4) | ((i > nph // 2) & (i <= nph // 2 + npback // 4))
          | ((i > nph) & (i <= nph + npback // 4))
          | ((i > 3 * nph // 2) & (i <= 3 * nph // 2 + npback // 4)))
    for s, key in ((0, "mean_vz_sheet1_electrons"), (1, "mean_vz_sheet1_ions")):
        sheet1 = np.tile(~bg, setup.nproc) & (st.parts[s][1] < ny / 2)
        assert round(st.parts[s][4][sheet1].mean(), 4) == pytest.approx(gold[key], abs=1e-12)
    # curnt, then the fold of fields at it = 1: jzm in the two central rows
    st.curnt()
    f = oracle_lib.fold(params, st.fld)
    jz = f[oracle_lib.JZM][[ny // 4, ny // 4 + 1], 1:nx + 1].mean()
    bx, by = f[oracle_lib.BX], f[oracle_lib.BY]
    rows = [ny // 4, ny // 4 + 1]
    curl = np.mean([((by[r, 2:nx + 2] - by[r, 1:nx + 1]) / params.dx
                     - (bx[r + 1, 1:nx + 1] - bx[r, 1:nx + 1]) / params.dy).mean()
                    for r in rows])
    assert round(jz, 3) == pytest.approx(gold["jz_deposited_central_cells"], abs=1e-12)
    assert round(curl, 3) == pytest.approx(gold["jz_curl_b_central_cells"], abs=1e-12)


def test_oracle_golden_vectors(oracle_lib):
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    out = mg.run(*mg.small_case())
    gold = np.load(os.path.join(HERE, "golden", "oracle_small.npz"))
    assert set(gold.files) == set(out)
    for k in gold.files:
        np.testing.assert_array_equal(out[k], gold[k], err_msg=k)


def _small_harris(nx=64, ny=32, ppc=8, seed=3):
    import oracle
    from maccpic_b200 import loader
    cfg = loader.HarrisConfig(nx=nx, ny=ny, ppc=ppc, seed=seed)
    fld, parts = loader.initial_state(cfg)
    rp = cfg.run_params()
    op = oracle.Params(nx=nx, ny=ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, qm=rp.qm, q=rp.q,
                       dn=rp.dn, am=rp.am, isav=rp.isav)
    return op, fld, parts


def test_permutation_noise_floor(oracle_lib):
    """The oracle against itself with the particles in another order: the
    floor under every parity tolerance of the GPU tests."""
    op, fld, parts = _small_harris()
    a = oracle_lib.State(op, fld, parts)
    rng = np.random.default_rng(0)
    perm = [rng.permutation(p.shape[1]) for p in parts]
    b = oracle_lib.State(op, fld, [p[:, q] for p, q in zip(parts, perm)])
    for _ in range(30):
        a.step()
        b.step()
    for k in range(6):
        err = np.abs(a.fld[k] - b.fld[k]).max() / np.abs(a.fld[k]).max()
        assert err < 1e-11, (k, err)


def test_single_particle_charge_and_weights(oracle_lib):
    """One particle deposits exactly q*dn/(dx dy) of charge after the fold,
    for positions on nodes, on cell centres and next to the wrap."""
    op = oracle_lib.Params(nx=8, ny=8, dx=0.5, dy=0.5, dt=0.05, qm=[-1.0], q=[-0.25],
                           dn=[1.0], am=[0.25], nsp=1)
    qd = -0.25 / 0.25
    for (x, y) in [(3.0, 4.0), (3.5, 2.5), (0.0, 0.0), (7.99, 7.99), (0.49, 7.51)]:
        part = np.array([[x], [y], [0.0], [0.0], [0.0], [1.0]])
        st = oracle_lib.State(op, np.zeros((13, 11, 11)), [part])
        st.curnt()
        f = oracle_lib.fold(op, st.fld)
        rho = f[oracle_lib.RHO][1:9, 1:9]
        assert rho.sum() == pytest.approx(qd, rel=1e-14)
        assert (rho <= 1e-300).all()  # negative charge only


def test_boris_rotation_conserves_energy(oracle_lib):
    """E = 0, uniform B: move leaves |u| (and gamma) unchanged and rotates
    the perpendicular momentum by the Boris angle -2 atan(qm B dt / 2 gamma)
    (counter-clockwise for an electron in +Bz)."""
    nx = ny = 8
    op = oracle_lib.Params(nx=nx, ny=ny, dx=0.5, dy=0.5, dt=0.05, qm=[-1.0], q=[-0.25],
                           dn=[1.0], am=[0.25], nsp=1)
    fld = np.zeros((13, ny + 3, nx + 3))
    bz = 0.7
    fld[oracle_lib.BZ] = bz
    u0 = np.array([0.3, -0.2, 0.1])
    g0 = np.sqrt(1 + (u0 ** 2).sum())
    part = np.array([[2.3], [5.6], [u0[0] / g0], [u0[1] / g0], [u0[2] / g0], [g0]])
    st = oracle_lib.State(op, fld, [part])
    st.move()
    v = st.parts[0][2:5, 0]
    g = st.parts[0][5, 0]
    assert g == pytest.approx(g0, rel=1e-14)
    u = v * g
    ang = np.arctan2(u[1], u[0]) - np.arctan2(u0[1], u0[0])
    t = -1.0 * bz * 0.05 / 2 / g0
    assert np.mod(ang, 2 * np.pi) == pytest.approx(np.mod(-2 * np.arctan(t), 2 * np.pi), rel=1e-12)
    assert u[2] == pytest.approx(u0[2], rel=1e-14)


def test_smooth2_transfer_function(oracle_lib):
    """smooth2 of a periodic Fourier mode returns the mode times
    (1+cos kx)(1+cos ky)/4 * (20 - 2cos kx - 2cos ky - 4 cos kx cos ky)/12."""
    nx, ny = 32, 16
    op = oracle_lib.Params(nx=nx, ny=ny, dx=0.5, dy=0.5, dt=0.05, qm=[-1.0], q=[-1.0],
                           dn=[1.0], am=[1.0], nsp=1)
    for mx, my in [(1, 0), (3, 2), (5, 7), (16, 8)]:
        kx, ky = 2 * np.pi * mx / nx, 2 * np.pi * my / ny
        ix = np.arange(nx + 3)[None, :]
        iy = np.arange(ny + 3)[:, None]
        a = np.cos(kx * ix + ky * iy)
        out = oracle_lib.smooth2(op, a)
        tb = (1 + np.cos(kx)) * (1 + np.cos(ky)) / 4
        tc = (20 - 2 * np.cos(kx) - 2 * np.cos(ky) - 4 * np.cos(kx) * np.cos(ky)) / 12
        np.testing.assert_allclose(out, a * tb * tc, atol=1e-13)


def test_poisson_cleans_divergence(oracle_lib):
    """After the Poisson correction div E - rho is at the CG tolerance."""
    nx, ny = 32, 24
    op = oracle_lib.Params(nx=nx, ny=ny, dx=0.5, dy=0.5, dt=0.05, qm=[-1.0], q=[-1.0],
                           dn=[1.0], am=[1.0], nsp=1)
    rng = np.random.default_rng(5)
    fld = np.zeros((13, ny + 3, nx + 3))
    rho = rng.normal(size=(ny, nx)) * 0.1
    rho -= rho.mean()
    fld[oracle_lib.RHO][1:ny + 1, 1:nx + 1] = rho
    # periodic guards as em2 keeps them
    r = fld[oracle_lib.RHO]
    r[:, 0], r[:, nx + 1], r[:, nx + 2] = r[:, nx], r[:, 1], r[:, 2]
    r[0, :], r[ny + 1, :], r[ny + 2, :] = r[ny, :], r[1, :], r[2, :]
    out, iters = oracle_lib.poisson(op, fld)
    ex, ey = out[oracle_lib.EX], out[oracle_lib.EY]
    div = ((ex[1:ny + 1, 1:nx + 1] - ex[1:ny + 1, 0:nx]) / 0.5
           + (ey[1:ny + 1, 1:nx + 1] - ey[0:ny, 1:nx + 1]) / 0.5 - rho)
    assert 1 <= iters < 10000
    assert np.mean((div * 0.25) ** 2) < 1e-9 * 1.01


def test_yee_vacuum_standing_wave_dispersion(oracle_lib):
    """Ez = cos(k x), B = 0 is a standing wave of the Yee scheme: after n
    calls Ez = cos(w n dt) cos(k x) with sin(w dt/2) = (c dt/dx) sin(k dx/2)."""
    nx, ny = 64, 4
    dx, dt = 0.5, 0.2
    op = oracle_lib.Params(nx=nx, ny=ny, dx=dx, dy=dx, dt=dt, qm=[-1.0], q=[-1.0],
                           dn=[1.0], am=[1.0], nsp=1)
    k = 2 * np.pi * 3 / (nx * dx)
    w = 2 / dt * np.arcsin(dt / dx * np.sin(k * dx / 2))
    fld = np.zeros((13, ny + 3, nx + 3))
    xe = (np.arange(nx + 3) - 0.5) * dx  # Ez(ix, iy) sits at x = (ix - 1/2) dx
    fld[oracle_lib.EZ] = np.cos(k * xe)[None, :]
    f = fld
    for n in range(1, 41):
        f = oracle_lib.yee(op, f)
        ez = f[oracle_lib.EZ][2, 1:nx + 1]
        a = (ez * np.cos(k * xe[1:nx + 1])).sum() * 2 / nx
        assert a == pytest.approx(np.cos(w * n * dt), abs=1e-12), n


def test_current_filter_known_answer(oracle_lib):
    """smooth_current = 1 filters each current array after the fold: from
    E = B = 0 and a single Fourier mode in jzm + jzp, Ez after fields is
    -dt/2 * (jzm + jzp) times smooth2's transfer function (1 with the filter
    off, as in em2).  Ez is untouched by the Poisson correction."""
    from oracle import EZ, JZM, JZP
    nx, ny = 32, 16
    mx, my = 3, 2
    kx, ky = 2 * np.pi * mx / nx, 2 * np.pi * my / ny
    tb = (1 + np.cos(kx)) * (1 + np.cos(ky)) / 4
    tc = (20 - 2 * np.cos(kx) - 2 * np.cos(ky) - 4 * np.cos(kx) * np.cos(ky)) / 12
    ix = np.arange(nx + 3)[None, :]
    iy = np.arange(ny + 3)[:, None]
    mode = np.cos(kx * ix + ky * iy)
    interior = (slice(1, ny + 1), slice(1, nx + 1))
    for flag, t in [(0, 1.0), (1, tb * tc)]:
        op = oracle_lib.Params(nx=nx, ny=ny, dx=0.5, dy=0.5, dt=0.05, qm=[-1.0], q=[-1.0],
                               dn=[1.0], am=[1.0], nsp=1, isav=1000, smooth_current=flag)
        fld = np.zeros((13, ny + 3, nx + 3))
        fld[JZM][interior] = mode[interior]          # guards zero: the fold adds nothing
        fld[JZP][interior] = 0.5 * mode[interior]
        st = oracle_lib.State(op, fld, [np.zeros((6, 0))])
        st.fields(1)
        np.testing.assert_allclose(st.fld[EZ][interior], -0.5 * op.dt * 1.5 * t * mode[interior],
                                   atol=1e-15)
