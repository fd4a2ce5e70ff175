"""The TMA-staged Yee and smooth2 stages (em2g_set_stencils(ctx, 1)) through
the C ABI.

FP64: bitwise equal to the oracle's smooth2 and to its Yee updates (the
stages round every cell as em2 does), and the whole em2g_fields call equal
to the direct-load stages' bit for bit.  FP32: the two implementations share
the per-cell arithmetic, so one em2g_fields call from the same state gives
the same bits.  Grids cover every residue of nx+3 mod 4 (each residue puts
the tiles' rows at other offsets inside the tensor map's 16-byte lines),
grids whose edges cut tiles, the last array of the field block (whose rows
reach the allocation's tail) and a grid with several tiles per persistent
CTA.  Inputs are random, guards included, so that em2's guard copies are
checked on values that are not periodic.
"""
import numpy as np
import pytest

from test_gpu_parity import harris_case, make_gpu, random_case, rel, TOL

pytestmark = pytest.mark.gpu

GRIDS = [(40, 24), (41, 25), (42, 26), (43, 31), (130, 70)]
NAMES = ["ex", "ey", "ez", "bx", "by", "bz", "rho", "jxm", "jxp", "jym", "jyp", "jzm", "jzp"]


@pytest.mark.parametrize("nx,ny", GRIDS + [(2048, 1024)])
def test_tma_smooth2_bitwise(gpu, oracle_lib, nx, ny):
    op, rp, fld, parts = random_case(nx=nx, ny=ny, n=64)
    rng = np.random.default_rng(nx * 7 + ny)
    with make_gpu(rp, fld, parts) as g:
        g.set_stencils(1)
        assert g.stencils() == 1
        for name in ("rho", "ex", "bz", "jzp"):  # jzp: the block's last array
            a = rng.normal(size=(ny + 3, nx + 3))
            g.set_field(name, a)
            g.smooth2(name)
            np.testing.assert_array_equal(g.get_field(name), oracle_lib.smooth2(op, a),
                                          err_msg=name)


@pytest.mark.parametrize("nx,ny", GRIDS)
@pytest.mark.parametrize("it", [1, 2])
def test_tma_fields_bitwise(gpu, oracle_lib, nx, ny, it):
    """As the direct-load test of the drop-in fields call: Bx, By, Bz, Ez
    bitwise against the oracle, Ex, Ey through the CG within tolerance; and
    every array bitwise equal to the direct-load stages' result."""
    op, rp, fld, parts = random_case(nx=nx, ny=ny, n=64, isav=2)
    rng = np.random.default_rng(3 + nx)
    fld = fld.copy()
    fld[6:] = 0.0
    fld[6:, 1:ny + 1, 1:nx + 1] = rng.normal(scale=0.01, size=(7, ny, nx))
    fld[6, 1:ny + 1, 1:nx + 1] -= fld[6, 1:ny + 1, 1:nx + 1].mean()
    st = oracle_lib.State(op, fld, parts)
    n_ref, _ = st.fields(it)
    out = []
    for mode in (1, 0):
        with make_gpu(rp, fld, parts) as g:
            g.set_stencils(mode)
            n, _ = g.fields(it)
            assert n == n_ref
            out.append(g.get_fields())
    got, direct = out
    for k in (2, 3, 4, 5):
        np.testing.assert_array_equal(got[k], st.fld[k], err_msg=str(k))
    for k in (0, 1):
        assert rel(got[k], st.fld[k]) < TOL, k
    np.testing.assert_array_equal(got, direct)


@pytest.mark.parametrize("nx,ny", [(40, 24), (43, 31), (130, 70)])
def test_tma_fp32_fields_equal_direct(gpu, nx, ny):
    """FP32: one fields call (with the current filter on, so that J goes
    through the staged smooth2 too) from one state, both implementations."""
    from maccpic_b200 import _lib
    from maccpic_b200.em2 import Em2Gpu
    op, rp, fld, parts = harris_case(nx=nx, ny=ny, ppc=4)
    rng = np.random.default_rng(5)
    fld = fld.copy()
    fld[6:, 1:ny + 1, 1:nx + 1] = rng.normal(scale=0.01, size=(7, ny, nx))
    rp.precision = _lib.FP32
    rp.smooth_current = 1
    rp.isav = 1  # E and B filtered too
    out = []
    for mode in (1, 0):
        with Em2Gpu(rp) as g:
            g.set_fields(fld)
            for s, p in enumerate(parts):
                g.set_particles(s, p)
            g.set_stencils(mode)
            g.fields(1)
            out.append(g.get_fields())
    np.testing.assert_array_equal(out[0], out[1])


def test_tma_steps_match_the_oracle(gpu, oracle_lib):
    """20 fused FP64 steps with the staged stages against the oracle (the
    deposit's atomics order is the only difference: 1e-10)."""
    op, rp, fld, parts = harris_case(nx=64, ny=32, ppc=16)
    st = oracle_lib.State(op, fld, parts)
    with make_gpu(rp, fld, parts) as g:
        g.set_stencils(1)
        for _ in range(20):
            r_ref = st.step()
            r = g.step(1)
            assert r["cg_iters"] == r_ref["cg_iters"]
        got = g.get_fields()
    for k in range(6):
        assert rel(got[k], st.fld[k]) < TOL, NAMES[k]


def test_stencil_mode_is_checked(gpu):
    from maccpic_b200 import _lib
    op, rp, fld, parts = random_case(n=16)
    with make_gpu(rp, fld, parts) as g:
        assert g.stencils() in (0, 1)
        with pytest.raises(Exception):
            g.set_stencils(2)
        L = _lib.lib()
        assert L.em2g_set_stencils(g._h, -1) == _lib.ERR_INVALID
