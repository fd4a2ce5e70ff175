"""The mixed-precision path (FP32 particles, gather, deposit, Yee; FP64
reductions) against the FP64 oracle.  FP32 arithmetic cannot be bitwise; the
bounds below are the ones the mixed path is held to:
  * positions round-trip through the cell-relative FP32 layout to < 2e-7
    cells, velocities to < 1e-6 relative;
  * after 50 steps of the double-Harris workload the field energy differs
    from the FP64 oracle's by < 1e-4 relative and E, B by < 1e-2 of their
    max |value| (the north-star target is 1e-3 on the field energy).
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
