"""The run diagnostics the GPU computes in FP64 (em2g_diagnostics), the files
written from them, and the GPU particle sampler, each against a host
computation.

* energies: 0.5 * mean over the interior of each of Ex..Bz squared
  (pic/fields.f90:267-347 over the whole grid), from the downloaded fields;
* reconnected flux of both sheets: max - min of psi = -integral of By dx
  along each sheet's centre row, from the downloaded By;
* Poisson residuals: mean r^2 of the last cgm before its first iteration
  and at exit (pic/fields.f90:546-616), against the oracle's cgm after the
  same steps (FP64: the stencils are bitwise equal, only the dot products'
  summation order differs);
* ene001.hst and the cf-p1 Bz frame written by maccpic_b200.output from a GPU
  run, read back against the downloaded arrays (pic/output.f90:151-199);
* the GPU sampler (torch Philox) against the host sampler (numpy Philox):
  the same counts and, within sampling error, the same moments.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def host_flux(by, nx, ny, dx, row):
    b = 0.5 * (by[row, 1:nx + 1] + by[row + 1, 1:nx + 1])
    psi = -np.cumsum(b) * dx
    return psi.max() - psi.min()


def host_energies(fld, nx, ny):
    a = fld[:6, 1:ny + 1, 1:nx + 1]
    return 0.5 * np.sum(a * a, axis=(1, 2)) / (nx * ny)


def _setup(precision, nx=96, ny=64, ppc=8, seed=4):
    import oracle
    from maccpic_b200 import loader
    cfg = loader.HarrisConfig(nx=nx, ny=ny, ppc=ppc, seed=seed)
    fld, parts = loader.initial_state(cfg)
    rp = cfg.run_params(precision=precision)
    op = oracle.Params(nx=nx, ny=ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, qm=rp.qm, q=rp.q, dn=rp.dn,
                       am=rp.am, isav=rp.isav)
    return cfg, rp, op, fld, parts


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_diagnostics_match_host_and_oracle(gpu, oracle_lib, precision):
    from maccpic_b200.em2 import Em2Gpu
    cfg, rp, op, fld, parts = _setup(precision)
    st = oracle_lib.State(op, fld, parts)
    with Em2Gpu(rp) as g:
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        for k in range(7):
            r = g.step(1)
            r_ref = st.step()
            assert r["cg_iters"] >= 1
        d = g.diagnostics()
        f = g.get_fields()
    nx, ny = cfg.nx, cfg.ny
    # FP64 sums over the same values (FP32 fields are exact in FP64): only
    # the summation order differs
    np.testing.assert_allclose(d["energies"], host_energies(f, nx, ny), rtol=1e-12, atol=0)
    for k, row in enumerate((ny // 4, ny // 4 + ny // 2)):
        np.testing.assert_allclose(d["flux"][k], host_flux(f[4], nx, ny, cfg.dx, row),
                                   rtol=1e-11)
    assert d["flux"][0] > 0 and d["flux"][1] > 0
    before, after = oracle_lib.last_cg_residuals()
    # cgm stopped at em2's test (pic/fields.f90:616), from a nonzero residual
    assert 0 <= d["poisson_r2_after"] < rp.cg_eps
    assert d["poisson_r2_before"] > 0
    if precision == 0:
        assert r["cg_iters"] == r_ref["cg_iters"]
        np.testing.assert_allclose(d["poisson_r2_before"], before, rtol=1e-9)
        np.testing.assert_allclose(d["poisson_r2_after"], after, rtol=1e-6)
        # and the energies of the oracle's fields, computed the same way
        np.testing.assert_allclose(d["energies"], host_energies(st.fld, nx, ny), rtol=1e-10)
    else:
        # the mixed path's charge-conservation residual tracks the FP64 one
        assert abs(np.log10(d["poisson_r2_before"] / before)) < 1.0


def test_output_files_from_a_gpu_run(gpu, tmp_path):
    """em2's ene###.hst line and cf-p1 Bz frame, written on the worker thread
    from a GPU run's diagnostics and downloads (pic/output.f90:151-199)."""
    from maccpic_b200.em2 import Em2Gpu
    from maccpic_b200.output import Em2Output
    cfg, rp, op, fld, parts = _setup(0, nx=64, ny=32, ppc=4)
    anme = parts[0].shape[1] * rp.am[0]      # pic/init.f90:119 with one rank
    out = Em2Output(str(tmp_path), cfg.nx, cfg.ny, rp.dt, anme)
    lines, bz100 = [], None
    with Em2Gpu(rp) as g:
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        for it in range(1, 101):
            ake = g.move_curnt()
            out.output(g, it, ake, isav=rp.isav)
            if it == 1 or it % rp.isav == 0:
                e = g.diagnostics()["energies"]
                lines.append([it * rp.dt, *e, *(ake / anme), e.sum() + (ake / anme).sum()])
            if it == 100:
                bz100 = g.get_field("bz")
            g.fields(it + 1)      # em2: output(it), it = it + 1, fields
    out.close()
    text = (tmp_path / "ene001.hst").read_text().splitlines()
    assert len(text) == len(lines) == 6
    for ln, want in zip(text, lines):
        vals = [float(ln[k:k + 13]) for k in range(0, len(ln.rstrip()), 13)]
        # e13.5 keeps five significant digits: half a unit of the fifth
        # digit is up to 5e-5 of the value
        np.testing.assert_allclose(vals, want, rtol=5e-5, atol=1e-300)
    frame = np.frombuffer((tmp_path / "cf-p1_001.bin").read_bytes(), "<f8")
    assert frame.size == 2 * bz100.size                    # frame 1 of file 001
    np.testing.assert_array_equal(frame[bz100.size:], bz100.ravel())
    prof = (tmp_path / "bz001.hst").read_text().splitlines()
    assert len(prof) == 6 and len(prof[0]) == cfg.ny * 13


def test_gpu_sampler_matches_host_sampler(gpu):
    """Both samplers draw the same double-Harris distribution: equal particle
    counts, equal sheet/background split, moments equal within sampling
    error (n = 2^21 per species)."""
    import torch
    from maccpic_b200 import loader
    cfg = loader.HarrisConfig(nx=256, ny=128, ppc=64, seed=3)
    host = loader.sample_particles(cfg)
    dev = [p.cpu().numpy() for p in loader.sample_particles_torch(cfg, device="cuda")]
    n = cfg.nx * cfg.ny * cfg.ppc
    te, ti = cfg.temperatures()
    for s in range(2):
        a, b = host[s], dev[s]
        assert a.shape == b.shape == (6, n)
        assert np.isfinite(b).all()
        assert (b[0] >= 0).all() and (b[0] < cfg.nx).all()
        assert (b[1] >= 0).all() and (b[1] < cfg.ny).all()
        # electrons and ions share positions in both samplers
        np.testing.assert_array_equal(dev[0][:2], dev[1][:2])
        # density profile in y: histograms over 32 bands agree to ~4 sigma
        ha = np.histogram(a[1], bins=32, range=(0, cfg.ny))[0]
        hb = np.histogram(b[1], bins=32, range=(0, cfg.ny))[0]
        assert (np.abs(ha - hb) <= 6 * np.sqrt(ha + 1)).all()
        # uniform in x
        assert abs(b[0].mean() / cfg.nx - 0.5) < 2e-3
        # gamma consistent with v
        v2 = b[2] ** 2 + b[3] ** 2 + b[4] ** 2
        np.testing.assert_allclose(b[5], 1 / np.sqrt(1 - v2), rtol=1e-12)
        # thermal spread of the transverse velocity, and the sheets' drift
        sd_a, sd_b = a[2].std(), b[2].std()
        assert abs(sd_b / sd_a - 1) < 5e-3
        for centre in (cfg.ny / 4, 3 * cfg.ny / 4):
            ma = np.abs(a[1] - centre) < 0.5
            mb = np.abs(b[1] - centre) < 0.5
            assert abs(mb.sum() - ma.sum()) < 6 * np.sqrt(ma.sum())
            err = 5 * sd_a / np.sqrt(ma.sum())
            assert abs(b[4][mb].mean() - a[4][ma].mean()) < err
    torch.cuda.empty_cache()
