"""The bounds-checked build of the FP32 push (libem2g_checked.so: the push's
units compiled with -DEM2G_BOUNDS_CHECK).  Every shared- and global-memory
index the push computes is checked before its access; one out of range is
counted and skipped, and the step then fails with EM2G_ERR_RANGE -- no trap
and no fault.

The runs below drive the push's index paths: particles on nodes, half
nodes and a hair below the box edges; the global-memory gather across the
periodic boundary; in-place pushes whose particles drift out of their group
cells (the deposit stack and its drain); regrouping pushes (the back-fill
written by the drain); grids whose last row segment is short; every compiled
variant; and an ensemble of uneven runs.  None may report an access out of
range, and each must give what the ordinary library gives (the deposit's
atomics order aside: FP32 round-off).
"""
import numpy as np
import pytest

from test_gpu_parity import harris_case, random_case, rel

pytestmark = pytest.mark.gpu


def _run(rp, fld, parts, library, steps, variant=None, interval=1):
    from maccpic_b200.em2 import Em2Gpu
    with Em2Gpu(rp, library=library) as g:
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        if variant is not None:
            g.set_variant(variant)
        g.set_sort_interval(min(interval, g.max_sort_interval()))
        out = g.step(steps)  # raises on an access out of range (EM2G_ERR_RANGE)
        return out, g.get_fields(), [g.get_particles(s) for s in range(len(parts))]


def _same(a, b):
    (ra, fa, pa), (rb, fb, pb) = a, b
    np.testing.assert_allclose(ra["ake"], rb["ake"], rtol=1e-5)
    for k in range(6):
        assert rel(fa[k], fb[k]) < 1e-4, k
    for x, y in zip(pa, pb):
        np.testing.assert_allclose(x, y, rtol=0, atol=1e-4)


@pytest.mark.parametrize("interval", [1, 3])
def test_checked_push_random_particles_at_edges(gpu, interval):
    from maccpic_b200 import _lib
    op, rp, fld, parts = random_case(nx=40, ny=24, n=5000)  # 40: a short last segment
    rp.precision = _lib.FP32
    got = _run(rp, fld, parts, _lib.checked_lib(), 12, interval=interval)
    want = _run(rp, fld, parts, _lib.lib(), 12, interval=interval)
    _same(got, want)


def test_checked_push_every_variant(gpu):
    from maccpic_b200 import _lib
    op, rp, fld, parts = harris_case(nx=96, ny=48, ppc=16)
    rp.precision = _lib.FP32
    from maccpic_b200.em2 import Em2Gpu
    with Em2Gpu(rp) as g:
        nvar = g.num_variants()
    for v in range(nvar):
        for interval in (1, 3):
            got = _run(rp, fld, parts, _lib.checked_lib(), 7, variant=v, interval=interval)
            want = _run(rp, fld, parts, _lib.lib(), 7, variant=v, interval=interval)
            _same(got, want)


def test_checked_push_ensemble(gpu):
    from maccpic_b200 import _lib, loader
    from maccpic_b200.ensemble import Em2Ensemble
    cfgs = [loader.HarrisConfig(nx=64, ny=32, ppc=8, seed=1),
            loader.HarrisConfig(nx=72, ny=40, ppc=4, seed=2, mass_ratio=49.0),
            loader.HarrisConfig(nx=128, ny=64, ppc=6, seed=3, mass_ratio=100.0, isav=5)]
    states = [(loader.initial_fields(c), loader.sample_particles(c)) for c in cfgs]
    res = []
    for library in (_lib.checked_lib(), _lib.lib()):
        runs = [c.run_params(np_max=[p[0].shape[1]] * 2, precision=_lib.FP32)
                for c, (_, p) in zip(cfgs, states)]
        with Em2Ensemble(runs, library=library) as e:
            for r, (fld, parts) in enumerate(states):
                e.set_fields(r, fld)
                for s, p in enumerate(parts):
                    e.set_particles(r, s, p)
            e.set_sort_interval(2)
            out = e.step(8)  # raises on an access out of range
            res.append((out, [e.get_fields(r) for r in range(len(cfgs))]))
    (oa, fa), (ob, fb) = res
    np.testing.assert_allclose(oa["ake"], ob["ake"], rtol=1e-5)
    for r in range(len(cfgs)):
        for k in range(6):
            assert rel(fa[r][k], fb[r][k]) < 1e-4, (r, k)
