"""Particle copies in slices (em2g_particles_begin / add / end and
em2g_get_particles_range): the path every particle upload and download now
takes, so that no device buffer grows with the particle count.  With a
small staging buffer (params.staging_mib = 1: 13k particles per host slice,
32k records per regrouping window) the 200k-particle species below goes
through many slices and windows.  Checked, for both precisions:

* an upload in uneven host slices, in device slices, and in one piece all
  give the same particles back (bitwise), and the same step afterwards;
* ranges read back equal the matching columns of the whole read, into host
  and into device arrays;
* a rejected slice (a non-finite value, a position outside the grid), an
  upload ended early, and slices out of order all leave the species'
  particles as they were.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(precision, staging_mib=1):
    from maccpic_b200 import loader
    cfg = loader.HarrisConfig(nx=128, ny=64, ppc=24, seed=11)
    fld, parts = loader.initial_state(cfg)
    rp = cfg.run_params(precision=precision, staging_mib=staging_mib)
    return cfg, rp, fld, parts


def _slices(p, cuts):
    edges = [0] + list(cuts) + [p.shape[1]]
    return [p[:, a:b] for a, b in zip(edges[:-1], edges[1:])]


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_slices_equal_one_piece(gpu, precision):
    import torch
    from maccpic_b200.em2 import Em2Gpu
    cfg, rp, fld, parts = _case(precision)
    n = parts[0].shape[1]
    cuts = [1, 5000, 77777, 150001]
    got = []
    for mode in ("whole", "host", "device"):
        with Em2Gpu(rp) as g:
            g.set_fields(fld)
            for s, p in enumerate(parts):
                if mode == "whole":
                    g.set_particles(s, p)
                elif mode == "host":
                    g.set_particles_slices(s, n, _slices(p, cuts))
                else:
                    g.set_particles_slices(s, n, [torch.from_numpy(np.ascontiguousarray(a)).cuda()
                                                  for a in _slices(p, cuts)])
            back = [g.get_particles(s) for s in range(2)]
            r = g.step(3)
            got.append((back, g.get_fields(), r["ake"]))
    for back, f, ake in got[1:]:
        for s in range(2):
            np.testing.assert_array_equal(back[s], got[0][0][s])
        # the deposits' atomics may add in another order (FP32: that round-off,
        # grown over three steps, is ~2e-5 of the largest value)
        tol = 1e-12 if precision == 0 else 1e-4
        for k in range(6):
            scale = max(np.abs(got[0][1][k]).max(), 1e-300)
            assert np.abs(f[k] - got[0][1][k]).max() / scale < tol, k
        np.testing.assert_allclose(ake, got[0][2], rtol=tol)
    if precision == 0:  # FP64 keeps the values themselves
        for s in range(2):
            np.testing.assert_array_equal(got[0][0][s], parts[s])


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_ranges_equal_the_whole_read(gpu, precision):
    import torch
    from maccpic_b200.em2 import Em2Gpu
    cfg, rp, fld, parts = _case(precision)
    with Em2Gpu(rp) as g:
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        g.step(2)
        n = parts[0].shape[1]
        for s in range(2):
            whole = g.get_particles(s)
            for a, b in ((0, n), (0, 1), (n - 1, n), (12345, 98765), (40000, 200000)):
                b = min(b, n)
                np.testing.assert_array_equal(g.get_particles_range(s, a, b - a), whole[:, a:b])
                dev = torch.empty((6, b - a), dtype=torch.float64, device="cuda")
                g.get_particles_range(s, a, b - a, out=dev)
                np.testing.assert_array_equal(dev.cpu().numpy(), whole[:, a:b])
        from maccpic_b200._lib import Em2gError, ERR_RANGE
        with pytest.raises(Em2gError) as ei:
            g.get_particles_range(0, n - 5, 10)
        assert ei.value.status == ERR_RANGE


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_rejected_or_incomplete_uploads_keep_the_particles(gpu, precision):
    from maccpic_b200 import _lib
    from maccpic_b200._lib import Em2gError
    from maccpic_b200.em2 import Em2Gpu
    cfg, rp, fld, parts = _case(precision)
    n = parts[0].shape[1]
    with Em2Gpu(rp) as g:
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        before = g.get_particles(0)
        for bad_value, status in ((np.nan, _lib.ERR_NONFINITE), (cfg.nx + 0.75, _lib.ERR_RANGE)):
            q = parts[0].copy()
            q[0 if status == _lib.ERR_RANGE else 4, 170000] = bad_value
            with pytest.raises(Em2gError) as ei:
                g.set_particles_slices(0, n, _slices(q, [60000, 120000]))
            assert ei.value.status == status
            np.testing.assert_array_equal(g.get_particles(0), before)
        # ended before every slot arrived
        with pytest.raises(Em2gError) as ei:
            g.set_particles_slices(0, n, _slices(parts[0], [60000])[:1])
        assert ei.value.status == _lib.ERR_INVALID
        np.testing.assert_array_equal(g.get_particles(0), before)
        # slices out of slot order
        L = g._L
        import ctypes as C
        _lib.check(L.em2g_particles_begin(g._h, 0, n))
        a = np.ascontiguousarray(parts[0][:, 100:200])
        rc = L.em2g_particles_add(g._h, 0, 100, 100, *[C.c_void_p(a[k].ctypes.data)
                                                       for k in range(6)], 0)
        assert rc == _lib.ERR_INVALID
        assert L.em2g_particles_end(g._h, 0) == _lib.ERR_INVALID
        np.testing.assert_array_equal(g.get_particles(0), before)
        # and the species still steps as before
        g.step(1)
