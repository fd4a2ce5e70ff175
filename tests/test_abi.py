"""The C ABI: libem2g.so loads on a CPU-only machine and exports every
function include/em2g.h declares; host-only entry points work without a GPU."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(em2g_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_function():
    from maccpic_b200 import build, _lib
    build.build()
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert names <= set(_lib.EXPORTS), sorted(names - set(_lib.EXPORTS))


def test_params_struct_layout_matches_header():
    from maccpic_b200 import _lib
    L = _lib.lib()
    P = _lib.Em2gParams()
    assert L.em2g_params_init(C.byref(P)) == 0
    assert P.struct_size == C.sizeof(_lib.Em2gParams)
    assert L.em2g_abi_version() == 1
    assert (P.cg_maxits, P.cg_eps, P.isav, P.c, P.qme) == (10000, 1e-9, 20, 1.0, -1.0)


def test_invalid_params_rejected_without_gpu():
    """Parameter validation happens before any device call."""
    from maccpic_b200 import _lib
    L = _lib.lib()
    P = _lib.Em2gParams()
    L.em2g_params_init(C.byref(P))
    P.nx, P.ny = 2, 64
    h = C.c_void_p()
    assert L.em2g_create(C.byref(P), C.byref(h)) == _lib.ERR_INVALID
    assert b"nx and ny" in L.em2g_last_error()
    L.em2g_params_init(C.byref(P))
    P.nx, P.ny, P.dx, P.dy, P.dt = 16, 16, 0.5, 0.5, 0.6
    assert L.em2g_create(C.byref(P), C.byref(h)) == _lib.ERR_INVALID
    assert b"c*dt" in L.em2g_last_error()
    L.em2g_params_init(C.byref(P))
    P.struct_size = 12
    assert L.em2g_create(C.byref(P), C.byref(h)) == _lib.ERR_INVALID


def test_invalid_ensembles_rejected_without_gpu():
    """em2g_ens_create checks every run before any device call."""
    from maccpic_b200 import _lib
    L = _lib.lib()

    def runs(n, **kw):
        arr = (_lib.Em2gParams * n)()
        for k in range(n):
            L.em2g_params_init(C.byref(arr[k]))
            arr[k].nx, arr[k].ny, arr[k].dx, arr[k].dy, arr[k].dt = 32, 16, 0.5, 0.5, 0.05
            arr[k].precision = _lib.FP32
            arr[k].np_max[0] = arr[k].np_max[1] = 100
            for name, v in kw.items():
                setattr(arr[k], name, v)
        return arr

    h = C.c_void_p()
    assert L.em2g_ens_create(runs(1), 0, C.byref(h)) == _lib.ERR_INVALID
    assert L.em2g_ens_create(runs(129), 129, C.byref(h)) == _lib.ERR_INVALID
    assert L.em2g_ens_create(runs(2, precision=_lib.FP64), 2, C.byref(h)) == _lib.ERR_INVALID
    assert b"FP32" in L.em2g_last_error()
    assert L.em2g_ens_create(runs(2, energy_mode=1), 2, C.byref(h)) == _lib.ERR_INVALID
    a = runs(2)
    a[1].np_max[1] = 0
    assert L.em2g_ens_create(a, 2, C.byref(h)) == _lib.ERR_INVALID
    assert b"np_max" in L.em2g_last_error()
    a = runs(2)
    a[1].device = 1
    assert L.em2g_ens_create(a, 2, C.byref(h)) == _lib.ERR_INVALID
    # 81 runs of 2 species: 162 pairs
    assert L.em2g_ens_create(runs(81), 81, C.byref(h)) == _lib.ERR_INVALID
    assert b"pairs" in L.em2g_last_error()
    a = runs(1)
    a[0].np_max[0] = a[0].np_max[1] = 1 << 30
    assert L.em2g_ens_create(a, 1, C.byref(h)) == _lib.ERR_RANGE
    assert h.value is None


def test_harris_ensemble_draws_the_uneven_batch():
    from maccpic_b200.ensemble import harris_ensemble
    cfgs = harris_ensemble(64, seed=0)
    assert len(cfgs) == 64
    assert all(128 <= c.nx <= 1024 and c.ny * 2 == c.nx and c.nx % 16 == 0 for c in cfgs)
    assert all(16 <= c.ppc <= 64 for c in cfgs)
    assert {c.mass_ratio for c in cfgs} == {25.0, 49.0, 100.0}
    assert len({c.seed for c in cfgs}) == 64
    assert len({c.psi0_over_b0di for c in cfgs}) == 64
    # log-uniform: both ends of the range are populated
    assert min(c.nx for c in cfgs) < 256 and max(c.nx for c in cfgs) > 512
    assert harris_ensemble(64, seed=0) == cfgs


def test_sort_interval_rules_without_gpu():
    from maccpic_b200 import _lib
    L = _lib.lib()
    P = _lib.Em2gParams()
    h = C.c_void_p()
    L.em2g_params_init(C.byref(P))
    P.nx, P.ny, P.dx, P.dy, P.dt = 32, 16, 0.5, 0.5, 0.05
    P.sort_interval = 2                         # FP64 regroups every step
    assert L.em2g_create(C.byref(P), C.byref(h)) == _lib.ERR_INVALID
    assert b"FP32" in L.em2g_last_error()
    P.precision = _lib.FP32
    P.sort_interval = 10                        # 10 * c * dt = dx
    assert L.em2g_create(C.byref(P), C.byref(h)) == _lib.ERR_INVALID
    assert b"sort_interval" in L.em2g_last_error()
    P.sort_interval = -1
    assert L.em2g_create(C.byref(P), C.byref(h)) == _lib.ERR_INVALID


def _build_c_caller(tmp_path, cxx: bool):
    import subprocess
    from maccpic_b200 import build
    build.build()
    libdir = os.path.join(ROOT, "maccpic_b200")
    exe = str(tmp_path / ("abi_smoke_cxx" if cxx else "abi_smoke_c"))
    cc = ["g++", "-x", "c++", "-std=c++17"] if cxx else ["gcc", "-std=c11"]
    cmd = cc + ["-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                os.path.join(ROOT, "tests", "abi_smoke.c"), "-o", exe,
                "-L", libdir, "-Wl,-rpath," + libdir, "-l:libem2g.so", "-lm"]
    subprocess.run(cmd, check=True)
    return exe


def test_c_and_cxx_callers_without_gpu(tmp_path):
    """include/em2g.h compiles as C11 and C++17 and the library links from
    both; the host-only checks run without a GPU."""
    import subprocess
    for cxx in (False, True):
        exe = _build_c_caller(tmp_path, cxx)
        out = subprocess.run([exe, "cpu"], capture_output=True, text=True)
        assert out.returncode == 0 and out.stdout.strip() == "ok", out.stderr


@pytest.mark.gpu
def test_c_caller_runs_a_step(gpu, tmp_path):
    import subprocess
    exe = _build_c_caller(tmp_path, cxx=False)
    out = subprocess.run([exe, "gpu"], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stderr


def test_stream_handles_for_the_library():
    """torch's default stream has handle 0, which the library reads as "its
    own stream"; the wrappers hand over the legacy default stream's explicit
    handle instead, so that work really is ordered on torch's stream."""
    from maccpic_b200.em2 import CUDA_STREAM_LEGACY, stream_handle

    class FakeStream:
        def __init__(self, h):
            self.cuda_stream = h

    assert stream_handle(None).value is None
    assert stream_handle(FakeStream(0)).value == CUDA_STREAM_LEGACY
    assert stream_handle(FakeStream(0x1234)).value == 0x1234
    assert stream_handle(0x5678).value == 0x5678


def test_output_buffers_are_checked_without_gpu():
    """A caller's output buffer for get_fields / get_particles must be a
    writeable C-contiguous float64 array of the exact shape."""
    import numpy as np
    from maccpic_b200.em2 import _check_out

    _check_out(np.empty((6, 10)), (6, 10))
    bad = [np.empty((6, 9)), np.empty((6, 10), dtype=np.float32), np.empty((10, 6)).T,
           np.empty((6, 20))[:, ::2]]
    ro = np.empty((6, 10))
    ro.flags.writeable = False
    for b in bad + [ro, [[0.0] * 10] * 6]:
        with pytest.raises(ValueError):
            _check_out(b, (6, 10))
