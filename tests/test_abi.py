"""The C ABI: libem2g.so loads on a CPU-only machine and exports every
function include/em2g.h declares; host-only entry points work without a GPU."""
import ctypes as C
import os
import re

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
