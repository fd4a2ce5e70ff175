"""Parity of the CUDA FP64 path with the CPU oracle, through the C ABI.

Tolerances: particle arithmetic and the stencil sweeps (fold, Yee,
smooth2) are bitwise equal to the oracle's for equal inputs (both avoid FMA
contraction and keep em2's evaluation order).  What differs is the order of
summation in the deposit (atomics), the CG dot products and ake/energies;
for those the test bound is 1e-10 relative to the array's max |value|,
against a measured oracle-vs-oracle floor of ~1e-13 under permuted particle
order (tests/test_oracle.py::test_permutation_noise_floor).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    scale = max(np.abs(a).max(), np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale


def periodize(a):
    """Set the guard columns/rows of (ny+3, nx+3) arrays from the interior,
    as em2 keeps them (periodic images 0 <- n, n+1 <- 1, n+2 <- 2)."""
    a = a.copy()
    nx, ny = a.shape[-1] - 3, a.shape[-2] - 3
    a[..., :, 0], a[..., :, nx + 1], a[..., :, nx + 2] = a[..., :, nx], a[..., :, 1], a[..., :, 2]
    a[..., 0, :], a[..., ny + 1, :], a[..., ny + 2, :] = a[..., ny, :], a[..., 1, :], a[..., 2, :]
    return a


def random_case(nx=40, ny=24, n=5000, seed=11, isav=2):
    import oracle
    from maccpic_b200.em2 import RunParams
    rng = np.random.default_rng(seed)
    kw = dict(nx=nx, ny=ny, dx=0.5, dy=0.5, dt=0.05, qm=[-1.0, 1 / 25.0],
              q=[-0.02, 0.02], dn=[1.0, 1.0], am=[0.02, 0.5], isav=isav)
    op = oracle.Params(**kw)
    rp = RunParams(np_max=[n, n], **kw)
    fld = np.zeros((13, ny + 3, nx + 3))
    fld[:6] = periodize(rng.normal(scale=0.05, size=(6, ny + 3, nx + 3)))
    parts = []
    for s in range(2):
        x = rng.random(n) * nx
        y = rng.random(n) * ny
        # a few particles exactly on nodes, on half nodes and at the edges
        x[:6] = [0.0, 0.5, 1.0, nx - 1e-12, nx - 0.5, 3.0]
        y[:6] = [0.0, ny - 1e-12, 0.5, 2.0, ny - 0.5, 1.5]
        u = rng.normal(scale=0.3 if s == 0 else 0.05, size=(3, n))
        g = np.sqrt(1 + (u * u).sum(0))
        parts.append(np.vstack([x, y, u / g, g]))
    return op, rp, fld, parts


def harris_case(nx=128, ny=64, ppc=16, seed=0):
    import oracle
    from maccpic_b200 import loader
    cfg = loader.HarrisConfig(nx=nx, ny=ny, ppc=ppc, seed=seed)
    fld, parts = loader.initial_state(cfg)
    rp = cfg.run_params()
    op = oracle.Params(nx=nx, ny=ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, qm=rp.qm, q=rp.q,
                       dn=rp.dn, am=rp.am, isav=rp.isav)
    return op, rp, fld, parts


def make_gpu(rp, fld, parts):
    from maccpic_b200.em2 import Em2Gpu
    g = Em2Gpu(rp)
    g.set_fields(fld)
    for s, p in enumerate(parts):
        g.set_particles(s, p)
    return g


def test_state_roundtrip(gpu):
    op, rp, fld, parts = random_case()
    with make_gpu(rp, fld, parts) as g:
        np.testing.assert_array_equal(g.get_fields(), fld)
        for s in range(2):
            np.testing.assert_array_equal(g.get_particles(s), parts[s])
        g.set_field("bz", fld[5] * 2)
        np.testing.assert_array_equal(g.get_field("bz"), fld[5] * 2)


def test_move_is_bitwise(gpu, oracle_lib):
    op, rp, fld, parts = random_case()
    st = oracle_lib.State(op, fld, parts)
    ake_ref = st.move()
    with make_gpu(rp, fld, parts) as g:
        ake = g.move()
        for s in range(2):
            np.testing.assert_array_equal(g.get_particles(s), st.parts[s])
        np.testing.assert_allclose(ake, ake_ref, rtol=1e-13)


def test_curnt_positions_bitwise_deposit_within_tolerance(gpu, oracle_lib):
    op, rp, fld, parts = random_case()
    st = oracle_lib.State(op, fld, parts)
    st.curnt()
    with make_gpu(rp, fld, parts) as g:
        g.curnt()
        for s in range(2):
            np.testing.assert_array_equal(g.get_particles(s), st.parts[s])
        got = g.get_fields()
        np.testing.assert_array_equal(got[:6], st.fld[:6])
        for k in range(6, 13):
            assert rel(got[k], st.fld[k]) < 1e-13, k


@pytest.mark.parametrize("it", [1, 2])
def test_fields_stencils_bitwise_poisson_within_tolerance(gpu, oracle_lib, it):
    """fields with random rho/J: Bx, By, Bz, Ez are untouched by the
    Poisson correction and must be bitwise; Ex, Ey go through the CG."""
    op, rp, fld, parts = random_case(isav=2)
    rng = np.random.default_rng(3)
    fld = fld.copy()
    # unfolded deposits: interior values, zero guards; total charge zero so
    # that the periodic Poisson problem is solvable
    ny, nx = fld.shape[1] - 3, fld.shape[2] - 3
    fld[6:] = 0.0
    fld[6:, 1:ny + 1, 1:nx + 1] = rng.normal(scale=0.01, size=(7, ny, nx))
    fld[6, 1:ny + 1, 1:nx + 1] -= fld[6, 1:ny + 1, 1:nx + 1].mean()
    st = oracle_lib.State(op, fld, parts)
    n_ref, e_ref = st.fields(it)
    with make_gpu(rp, fld, parts) as g:
        n, e = g.fields(it)
        got = g.get_fields()
    for k in (2, 3, 4, 5):
        np.testing.assert_array_equal(got[k], st.fld[k], err_msg=str(k))
    assert n == n_ref
    for k in (0, 1):
        assert rel(got[k], st.fld[k]) < TOL, k
    np.testing.assert_array_equal(got[6:], 0.0)
    if it % 2 == 0:
        np.testing.assert_allclose(e, e_ref, rtol=1e-12)
    else:
        assert e is None


def test_smooth2_bitwise(gpu, oracle_lib):
    op, rp, fld, parts = random_case()
    with make_gpu(rp, fld, parts) as g:
        for name, k in (("rho", 6), ("ex", 0), ("bz", 5)):
            g.smooth2(name)
            np.testing.assert_array_equal(g.get_field(name), oracle_lib.smooth2(op, fld[k]))


def test_dropin_sequence_100_steps(gpu, oracle_lib):
    """move / curnt / fields through the ABI, as em2's main loop calls them."""
    op, rp, fld, parts = harris_case(nx=64, ny=32, ppc=16)
    st = oracle_lib.State(op, fld, parts)
    with make_gpu(rp, fld, parts) as g:
        for it in range(1, 101):
            ake_ref = st.move()
            st.curnt()
            n_ref, e_ref = st.fields(it)
            ake = g.move()
            g.curnt()
            n, e = g.fields(it)
            assert n == n_ref, it
            np.testing.assert_allclose(ake, ake_ref, rtol=1e-12)
            if e_ref is not None and it % rp.isav == 0:
                np.testing.assert_allclose(e, e_ref, rtol=1e-9)
        got = g.get_fields()
        for k in range(6):
            assert rel(got[k], st.fld[k]) < TOL, k
        for s in range(2):
            assert rel(g.get_particles(s), st.parts[s]) < 1e-12


def test_fused_step_parity_100_steps(gpu, oracle_lib):
    """The fused fast path (em2g_step) against the oracle's main loop on the
    double-Harris workload at 128x64, 16 particles per cell per species."""
    op, rp, fld, parts = harris_case(nx=128, ny=64, ppc=16)
    st = oracle_lib.State(op, fld, parts)
    with make_gpu(rp, fld, parts) as g:
        for k in range(100):
            r_ref = st.step()
            r = g.step(1)
            assert r["cg_iters"] == r_ref["cg_iters"], k
            np.testing.assert_allclose(r["ake"], r_ref["ake"], rtol=1e-12)
        got = g.get_fields()
        for k in range(6):
            assert rel(got[k], st.fld[k]) < TOL, k
        for s in range(2):
            assert rel(g.get_particles(s), st.parts[s]) < 1e-12


def test_invalid_particles_rejected(gpu):
    from maccpic_b200._lib import Em2gError, ERR_RANGE, ERR_NONFINITE
    op, rp, fld, parts = random_case(n=100)
    with make_gpu(rp, fld, parts) as g:
        bad = parts[0].copy()
        bad[0, 5] = rp.nx + 0.75
        with pytest.raises(Em2gError) as ei:
            g.set_particles(0, bad)
        assert ei.value.status == ERR_RANGE
        bad = parts[0].copy()
        bad[3, 7] = np.nan
        with pytest.raises(Em2gError) as ei:
            g.set_particles(0, bad)
        assert ei.value.status == ERR_NONFINITE
        with pytest.raises(Em2gError) as ei:
            g.set_particles(0, np.zeros((6, 101)))
        assert ei.value.status == ERR_RANGE
        # the context is still usable afterwards
        g.step(1)


def test_fast_path_deposit_matches_split_sum(gpu, oracle_lib):
    """em2g_move_curnt (cell-sorted fast path) against oracle move + curnt:
    particles bitwise, rho and jm+jp (kept in the jxm arrays) within TOL,
    jxp/jyp/jzp zero."""
    op, rp, fld, parts = random_case(n=20000)
    st = oracle_lib.State(op, fld, parts)
    ake_ref = st.move()
    st.curnt()
    with make_gpu(rp, fld, parts) as g:
        ake = g.move_curnt()
        for s in range(2):
            np.testing.assert_array_equal(g.get_particles(s), st.parts[s])
        got = g.get_fields()
    np.testing.assert_allclose(ake, ake_ref, rtol=1e-13)
    np.testing.assert_array_equal(got[:6], st.fld[:6])
    assert rel(got[6], st.fld[6]) < TOL
    for m, p in ((7, 8), (9, 10), (11, 12)):
        assert rel(got[m], st.fld[m] + st.fld[p]) < TOL, m
        np.testing.assert_array_equal(got[p], 0.0)


def test_fast_path_rows_beyond_the_box(gpu, oracle_lib):
    """em2's own loader can leave particles at y in [ny, ny+0.5) (its guard
    cells absorb them); the fast path must treat them as the oracle does."""
    op, rp, fld, parts = random_case(n=3000)
    parts = [p.copy() for p in parts]
    for p in parts:
        p[1, :200] = rp.ny + 0.49 * np.linspace(0, 1, 200, endpoint=False)
        p[0, 200:400] = rp.nx + 0.49 * np.linspace(0, 1, 200, endpoint=False)
    st = oracle_lib.State(op, fld, parts)
    with make_gpu(rp, fld, parts) as g:
        for it in range(1, 6):
            st.move()
            st.curnt()
            st.fields(it)
            g.move_curnt()
            g.fields(it)
        got = g.get_fields()
        for k in range(6):
            assert rel(got[k], st.fld[k]) < TOL, k
        for s in range(2):
            assert rel(g.get_particles(s), st.parts[s]) < 1e-12


def test_drop_in_and_fast_paths_interleave(gpu, oracle_lib):
    """Separate move/curnt calls (exact jm/jp split) and the fast path can be
    mixed on one context; the particle bookkeeping stays consistent."""
    op, rp, fld, parts = harris_case(nx=64, ny=32, ppc=8)
    st = oracle_lib.State(op, fld, parts)
    with make_gpu(rp, fld, parts) as g:
        for it in range(1, 13):
            st.move()
            st.curnt()
            st.fields(it)
            if it % 3 == 0:
                g.move()
                g.curnt()
            else:
                g.move_curnt()
            g.fields(it)
        got = g.get_fields()
        for k in range(6):
            assert rel(got[k], st.fld[k]) < TOL, k
        for s in range(2):
            assert rel(g.get_particles(s), st.parts[s]) < 1e-12


def test_gpu_restart_through_em2_files(gpu, tmp_path, oracle_lib):
    """Write em2's restart files from the GPU state after curnt, read them
    into a new context, run fields as cont does and carry on: the result
    matches the oracle's straight run within TOL."""
    from maccpic_b200 import dumpio
    op, rp, fld, parts = harris_case(nx=64, ny=32, ppc=8)
    st = oracle_lib.State(op, fld, parts)
    for it in range(1, 11):
        st.move()
        st.curnt()
        st.fields(it)
    with make_gpu(rp, fld, parts) as g:
        for it in range(1, 5):
            g.move_curnt()
            g.fields(it)
        g.move_curnt()
        dumpio.save(g, str(tmp_path))
    from maccpic_b200.em2 import Em2Gpu
    with Em2Gpu(rp) as h:
        dumpio.load(h, str(tmp_path), [p.shape[1] for p in parts])
        h.fields(5)
        for it in range(6, 11):
            h.move_curnt()
            h.fields(it)
        got = h.get_fields()
        for k in range(6):
            assert rel(got[k], st.fld[k]) < TOL, k
        for s in range(2):
            assert rel(h.get_particles(s), st.parts[s]) < 1e-12


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gpu_compact_checkpoint(gpu, tmp_path, precision):
    """dumpio.save_compact between full steps, load_compact into a new
    context: it carries on with the same step counter and, stepping on, ends
    where the context that was never stopped ends (FP64 bitwise in the
    particles; the deposit's atomics order aside, to round-off)."""
    from maccpic_b200 import _lib, dumpio
    from maccpic_b200.em2 import Em2Gpu
    op, rp, fld, parts = harris_case(nx=64, ny=32, ppc=8)
    if precision == "fp32":
        rp.precision = _lib.FP32
    path = str(tmp_path / "state.npz")
    with make_gpu(rp, fld, parts) as g:
        g.step(6)
        dumpio.save_compact(g, path)
        g.step(4)
        want_f, want_p = g.get_fields(), [g.get_particles(s) for s in range(2)]
    with Em2Gpu(rp) as h:
        dumpio.load_compact(h, path)
        assert h.it == 6
        h.step(4)
        assert h.it == 10
        got_f = h.get_fields()
        for k in range(6):
            assert rel(got_f[k], want_f[k]) < (1e-10 if precision == "fp64" else 1e-4), k
        for s in range(2):
            tol = 1e-12 if precision == "fp64" else 1e-4
            assert np.abs(h.get_particles(s) - want_p[s]).max() < tol


def test_every_push_variant_matches_the_oracle(gpu, oracle_lib):
    """The autotuner's kernel variants compute the same step."""
    from maccpic_b200.em2 import Em2Gpu
    op, rp, fld, parts = harris_case(nx=96, ny=32, ppc=8)
    st = oracle_lib.State(op, fld, parts)
    for _ in range(6):
        st.step()
    with Em2Gpu(rp) as probe:
        n = probe.num_variants()
    assert n >= 2
    for v in range(n):
        with make_gpu(rp, fld, parts) as g:
            g.set_variant(v)
            assert g.variant()[0] == v
            for _ in range(6):
                g.step(1)
            got = g.get_fields()
            for k in range(6):
                assert rel(got[k], st.fld[k]) < TOL, (v, k)
            for s in range(2):
                assert rel(g.get_particles(s), st.parts[s]) < 1e-12, v


def test_current_filter_matches_the_oracle(gpu, oracle_lib):
    """smooth_current = 1 (no em2 counterpart): the drop-in sequence, which
    deposits jm and jp separately, and the fused path, which deposits their
    sum, against the oracle with the same filter."""
    import dataclasses
    op, rp, fld, parts = harris_case(nx=64, ny=32, ppc=16)
    op = dataclasses.replace(op, smooth_current=1)
    rp = dataclasses.replace(rp, smooth_current=1)
    st_a = oracle_lib.State(op, fld, parts)
    st_b = st_a.copy()
    with make_gpu(rp, fld, parts) as a, make_gpu(rp, fld, parts) as b:
        for it in range(1, 31):
            st_a.move()
            st_a.curnt()
            n_ref, _ = st_a.fields(it)
            a.move()
            a.curnt()
            n, _ = a.fields(it)
            assert n == n_ref, it
            r_ref = st_b.step()
            r = b.step(1)
            assert r["cg_iters"] == r_ref["cg_iters"], it
        for g, st in ((a, st_a), (b, st_b)):
            got = g.get_fields()
            for k in range(6):
                assert rel(got[k], st.fld[k]) < TOL, k
            for s in range(2):
                assert rel(g.get_particles(s), st.parts[s]) < 1e-12


def species_moments(part, nx, ny, mass):
    """Per-species moments deposited by the harness (em2 has none): density,
    particle flux (n vx, n vy, n vz) and kinetic energy density on the
    cells, nearest-cell weighting."""
    x, y, vx, vy, vz, g = part
    cell = (np.floor(y).astype(np.int64) % ny) * nx + (np.floor(x).astype(np.int64) % nx)
    out = []
    for w in (np.ones_like(x), vx, vy, vz, mass * (g - 1.0)):
        out.append(np.bincount(cell, weights=w, minlength=nx * ny))
    return np.array(out)


def test_species_moments_after_100_steps(gpu, oracle_lib):
    op, rp, fld, parts = harris_case(nx=64, ny=32, ppc=16, seed=5)
    st = oracle_lib.State(op, fld, parts)
    with make_gpu(rp, fld, parts) as g:
        for _ in range(100):
            st.step()
        g.step(100)
        for s in range(2):
            m_gpu = species_moments(g.get_particles(s), op.nx, op.ny, rp.am[s])
            m_ref = species_moments(st.parts[s], op.nx, op.ny, rp.am[s])
            for k in range(5):
                assert rel(m_gpu[k], m_ref[k]) < 1e-10, (s, k)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_invalid_fields_leave_the_state(gpu, precision):
    """Field uploads are checked on the device before they replace anything:
    a non-finite value is refused and the fields stay as they were."""
    from maccpic_b200 import _lib
    from maccpic_b200._lib import Em2gError, ERR_NONFINITE
    import dataclasses
    op, rp, fld, parts = random_case(n=100)
    rp = dataclasses.replace(rp, precision=_lib.FP32 if precision == "fp32" else _lib.FP64)
    with make_gpu(rp, fld, parts) as g:
        before = g.get_fields()
        bad = fld.copy()
        bad[4, 3, 5] = np.inf
        with pytest.raises(Em2gError) as ei:
            g.set_fields(bad)
        assert ei.value.status == ERR_NONFINITE
        np.testing.assert_array_equal(g.get_fields(), before)
        bad = parts[1].copy()
        bad[2, 9] = np.nan
        with pytest.raises(Em2gError):
            g.set_particles(1, bad)
        g.step(1)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", ["vacuum", "pair"])
def test_empty_and_single_particle_species(gpu, oracle_lib, precision, case):
    """Species holding no particle ("vacuum": the fields alone) or a single
    one ("pair": one electron at x = nx - 1e-12, which FP32 rounds onto the
    next cell's edge, and one ion, so that the periodic Poisson problem stays
    solvable) step like the oracle on either path: the grouping, scans,
    pushes and copies at their empty and one-element edges.  FP64 to the
    file's tolerance, with the oracle's CG iteration counts; FP32 to the
    mixed path's bounds (tests/test_gpu_fp32.py: its CG may stop a few
    iterations apart, each solve meeting mean r^2 < 1e-9): 1e-3 of a field's
    max |value|, 1e-3 relative on ake and velocities, 1e-4 cells."""
    import dataclasses
    from maccpic_b200 import _lib
    op, rp, fld, parts = random_case(nx=40, ny=24, n=16)
    k = 0 if case == "vacuum" else 1
    parts = [parts[0][:, 3:3 + k].copy(), parts[1][:, 5:5 + k].copy()]
    fp32 = precision == "fp32"
    rp = dataclasses.replace(rp, np_max=[1, 1], precision=_lib.FP32 if fp32 else _lib.FP64)
    st = oracle_lib.State(op, fld, parts)
    with make_gpu(rp, fld, parts) as g:
        for s in range(2):
            assert g.get_particles(s).shape == (6, k)
        for _ in range(5):
            r_ref = st.step()
            r = g.step(1)
            assert r["cg_iters"] < 1000 and r_ref["cg_iters"] < 1000
            if not fp32:
                assert r["cg_iters"] == r_ref["cg_iters"]
            np.testing.assert_allclose(r["ake"], r_ref["ake"], rtol=1e-3 if fp32 else 1e-12)
        got = g.get_fields()
        for f in range(6):
            assert rel(got[f], st.fld[f]) < (1e-3 if fp32 else TOL), f
        n = np.array([[op.nx], [op.ny]])
        for s in range(2):
            p = g.get_particles(s)
            assert p.shape == (6, k)
            d = p[:2] - st.parts[s][:2]
            d -= n * np.round(d / n)
            assert d.size == 0 or np.abs(d).max() < (1e-4 if fp32 else 1e-12)
            np.testing.assert_allclose(p[2:], st.parts[s][2:], rtol=1e-3 if fp32 else 1e-12)
