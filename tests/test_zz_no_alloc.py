"""em2g_smooth2_static: smooth2 on a caller's device array without any
device allocation, for callers that cannot call cudaMalloc (they manage
their device memory themselves or are inside a stream capture) and so cannot
create an em2g context.  Its scratch is a fixed static device array shared
by all calls.  Checked against the context entry point em2g_smooth2 on two
calls in a row (different grids, so the shared scratch is reused), with the
tolerance of the FP64 stencil tests: bitwise equality.  Each result is also
checked bitwise against the oracle's smooth2, so the entry point is pinned
to em2's filter independently of the context path.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference_smooth(nx, ny, a):
    from maccpic_b200.em2 import RunParams, Em2Gpu
    rp = RunParams(nx=nx, ny=ny, dx=0.5, dy=0.5, dt=0.05, qm=[-1.0], q=[-1.0], dn=[1.0],
                   am=[1.0], np_max=[1], nsp=1)
    with Em2Gpu(rp) as g:
        g.set_field("rho", a)
        g.smooth2("rho")
        return g.get_field("rho")


def _static_smooth(nx, ny, t):
    import torch
    from maccpic_b200 import _lib
    st = torch.cuda.current_stream()
    rc = _lib.lib().em2g_smooth2_static(nx, ny, C.c_void_p(t.data_ptr()),
                                        C.c_void_p(st.cuda_stream))
    _lib.check(rc)
    torch.cuda.synchronize()


def _oracle_smooth(oracle, nx, ny, a):
    op = oracle.Params(nx=nx, ny=ny, dx=0.5, dy=0.5, dt=0.05, qm=[-1.0], q=[-1.0], dn=[1.0],
                       am=[1.0], nsp=1)
    return oracle.smooth2(op, a)


def test_static_smooth2_matches_context_entry_point(gpu, oracle_lib):
    import torch
    rng = np.random.default_rng(21)
    for nx, ny in ((40, 24), (96, 70)):       # two calls in a row, two grids
        a = rng.normal(size=(ny + 3, nx + 3))
        t = torch.from_numpy(a.copy()).cuda()
        _static_smooth(nx, ny, t)
        got = t.cpu().numpy()
        np.testing.assert_array_equal(got, _reference_smooth(nx, ny, a))
        np.testing.assert_array_equal(got, _oracle_smooth(oracle_lib, nx, ny, a))
    # and twice on the same array
    nx, ny = 33, 17
    a = rng.normal(size=(ny + 3, nx + 3))
    t = torch.from_numpy(a.copy()).cuda()
    _static_smooth(nx, ny, t)
    _static_smooth(nx, ny, t)
    once = _reference_smooth(nx, ny, a)
    np.testing.assert_array_equal(t.cpu().numpy(), _reference_smooth(nx, ny, once))


def test_static_smooth2_rejects_grids_beyond_its_scratch(gpu):
    import torch
    from maccpic_b200 import _lib
    L = _lib.lib()
    t = torch.zeros(8, device="cuda", dtype=torch.float64)
    rc = L.em2g_smooth2_static(1021, 1021, C.c_void_p(t.data_ptr()), None)
    assert rc == _lib.ERR_RANGE
    assert b"exceeds the static scratch" in L.em2g_last_error()
    assert L.em2g_smooth2_static(2, 64, C.c_void_p(t.data_ptr()), None) == _lib.ERR_INVALID
