"""Failure detection on the GPU without a fault: every wait of a device
thread on other threads is bounded, and a wait that runs out becomes a status
the host reads (EM2G_ERR_TIMEOUT from the next call), not a hang.

em2g_selftest_waits makes one wait of each kind run out on purpose -- the
CG's grid barrier, counted for one block more than arrive, and a TMA tile's
mbarrier that no copy completes -- and returns the statuses they recorded.
The context must then step exactly as before: its next steps are checked
against the oracle.
"""
import ctypes as C
import time

import numpy as np
import pytest

from test_gpu_parity import harris_case, make_gpu, rel, TOL

pytestmark = pytest.mark.gpu


def test_bounded_waits_run_out_and_leave_the_context_usable(gpu, oracle_lib):
    from maccpic_b200 import _lib
    op, rp, fld, parts = harris_case(nx=64, ny=32, ppc=8)
    st = oracle_lib.State(op, fld, parts)
    with make_gpu(rp, fld, parts) as g:
        cg, tma = C.c_int(-1), C.c_int(-1)
        t0 = time.perf_counter()
        _lib.check(_lib.lib().em2g_selftest_waits(g._h, C.byref(cg), C.byref(tma)))
        waited = time.perf_counter() - t0
        assert cg.value == 1, cg.value    # the grid barrier's bound ran out
        assert tma.value == 2, tma.value  # the tile wait's bound ran out
        assert 1.0 < waited < 30.0, waited  # bounded: seconds, not forever
        for _ in range(5):  # and nothing of the probes is left behind
            r_ref = st.step()
            r = g.step(1)
            assert r["cg_iters"] == r_ref["cg_iters"]
        got = g.get_fields()
    for k in range(6):
        assert rel(got[k], st.fld[k]) < TOL, k
