"""em2's start-up velocity push (pic/setv.f90:36-128) on the GPU,
em2g_setv_device: one Boris push of -dt/2 with linear weights.  Bitwise
against the oracle's restatement (em2o_setv) for both species, with E and B
of every component nonzero and the tx/ty background terms set, so that each
gather and each term of the rotation is exercised; particles on cell edges
and near the box's far edges included.  Bad input (outside the box, |v| >=
1, non-finite) is rejected and leaves the block as it was.  The loader's
start-up option applies the same push to GPU-drawn particles."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(seed=3, nx=48, ny=40, n=20000):
    from maccpic_b200.em2 import RunParams
    rng = np.random.default_rng(seed)
    rp = RunParams(nx=nx, ny=ny, dx=0.5, dy=0.5, dt=0.05, nsp=2, qm=[-1.0, 1.0 / 25.0],
                   q=[-0.01, 0.01], dn=[1.0, 1.0], am=[0.01, 0.25], tx=[0.003, -0.002],
                   ty=[-0.001, 0.004], np_max=[n, n])
    fld = np.zeros((13, ny + 3, nx + 3))
    fld[:6] = rng.normal(scale=0.3, size=(6, ny + 3, nx + 3))
    parts = []
    for s in range(2):
        p = np.zeros((6, n))
        p[0] = rng.uniform(0, nx, n)
        p[1] = rng.uniform(0, ny, n)
        # cell edges, half cells and the far edges of the box
        k = n // 10
        p[0, :k] = rng.integers(0, nx, k) + rng.choice([0.0, 0.5, 1 - 2**-40], k)
        p[1, :k] = rng.integers(0, ny, k) + rng.choice([0.0, 0.5, 1 - 2**-40], k)
        p[0, k:2 * k] = np.nextafter(nx, 0)
        v = rng.normal(scale=0.3 if s == 0 else 0.05, size=(3, n))
        sp = np.sqrt((v * v).sum(0))
        v[:, sp >= 0.95] *= 0.9 / sp[sp >= 0.95]
        p[2:5] = v
        p[5] = 1.0 / np.sqrt(1.0 - (v * v).sum(0))
        parts.append(p)
    return rp, fld, parts


def _oracle_params(oracle, rp):
    return oracle.Params(nx=rp.nx, ny=rp.ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, c=rp.c,
                         qm=rp.qm, q=rp.q, dn=rp.dn, am=rp.am, tx=rp.tx, ty=rp.ty, nsp=rp.nsp)


def test_setv_is_bitwise_the_oracles(gpu, oracle_lib):
    import torch
    from maccpic_b200.em2 import setv_device
    rp, fld, parts = _case()
    op = _oracle_params(oracle_lib, rp)
    fd = torch.from_numpy(fld).cuda()
    for s, p in enumerate(parts):
        ref = oracle_lib.setv(op, fld, s, p)
        t = torch.from_numpy(p).cuda()
        setv_device(rp, s, fd, t)
        got = t.cpu().numpy()
        np.testing.assert_array_equal(got, ref)
        assert not np.array_equal(got[2:], p[2:])   # the push did something


@pytest.mark.parametrize("bad", ["x_high", "y_negative", "speed_of_light", "nan"])
def test_setv_rejects_bad_particles_and_leaves_them(gpu, bad):
    import torch
    from maccpic_b200._lib import Em2gError
    from maccpic_b200.em2 import setv_device
    rp, fld, parts = _case(n=5000)
    p = parts[0].copy()
    j = 1234
    if bad == "x_high":
        p[0, j] = rp.nx
    elif bad == "y_negative":
        p[1, j] = -1e-12
    elif bad == "speed_of_light":
        p[2:5, j] = [0.6, 0.8, 0.0]
    else:
        p[3, j] = np.nan
    t = torch.from_numpy(p).cuda()
    with pytest.raises(Em2gError):
        setv_device(rp, 0, torch.from_numpy(fld).cuda(), t)
    np.testing.assert_array_equal(t.cpu().numpy(), p)


def test_loader_start_up_push_on_drawn_particles(gpu, oracle_lib):
    """loader.setv_torch on GPU-drawn particles equals the oracle's setv on
    the same draw, and the drawn positions are untouched."""
    from maccpic_b200 import loader
    cfg = loader.HarrisConfig(nx=64, ny=32, ppc=8, seed=5, psi0_over_b0di=0.1)
    fld = loader.initial_fields(cfg)
    fld[0] += 1e-3   # a uniform Ex, so that the E gathers contribute
    parts = loader.sample_particles_torch(cfg, device="cuda")
    before = [p.cpu().numpy() for p in parts]
    loader.setv_torch(cfg, fld, parts)
    rp = cfg.run_params()
    op = _oracle_params(oracle_lib, rp)
    for s, p in enumerate(parts):
        got = p.cpu().numpy()
        np.testing.assert_array_equal(got, oracle_lib.setv(op, fld, s, before[s]))
        np.testing.assert_array_equal(got[:2], before[s][:2])
