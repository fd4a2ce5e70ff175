"""ctypes binding of libem2g.so (the C ABI in include/em2g.h).

The library is built in-tree (``python -m maccpic_b200.build``); importing
this module never falls back to anything else: if the shared object is
missing or fails to load, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libem2g.so")
# the bounds-checked build of the same library (maccpic_b200/build.py)
LIB_CHECKED_PATH = os.path.join(PKG, "libem2g_checked.so")

MAX_SPECIES = 4
NFIELD = 13
FIELD_NAMES = ["ex", "ey", "ez", "bx", "by", "bz", "rho",
               "jxm", "jxp", "jym", "jyp", "jzm", "jzp"]
FIELD_ID = {n: i for i, n in enumerate(FIELD_NAMES)}

OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_RANGE, ERR_TIMEOUT, ERR_NONFINITE = range(7)
FP64, FP32 = 0, 1

# every entry point declared in include/em2g.h
EXPORTS = [
    "em2g_abi_version", "em2g_last_error", "em2g_params_init", "em2g_create",
    "em2g_destroy", "em2g_set_stream", "em2g_synchronize", "em2g_set_field",
    "em2g_get_field", "em2g_set_fields", "em2g_get_fields", "em2g_set_particles",
    "em2g_get_particles", "em2g_particles_begin", "em2g_particles_add", "em2g_particles_end",
    "em2g_get_particles_range", "em2g_set_step", "em2g_get_step", "em2g_set_fields_device",
    "em2g_get_fields_device", "em2g_field_device_ptr", "em2g_move", "em2g_curnt",
    "em2g_fields", "em2g_smooth2", "em2g_step", "em2g_set_particles_device",
    "em2g_move_curnt", "em2g_set_timing", "em2g_get_counters", "em2g_reset_counters",
    "em2g_smooth2_static", "em2g_setv_device", "em2g_diagnostics", "em2g_num_variants", "em2g_set_variant",
    "em2g_get_variant", "em2g_set_sort_interval", "em2g_set_stencils", "em2g_get_stencils",
    "em2g_selftest_waits",
    "em2g_adj_create", "em2g_adj_destroy", "em2g_adj_forward", "em2g_adj_keep_all_fields",
    "em2g_adj_field_slots", "em2g_adj_get_field_slots",
    "em2g_adj_seed_fields_device",
    "em2g_adj_backward", "em2g_adj_get_fields_device", "em2g_adj_get_particles_device",
    "em2g_adj_get_initial_particles_device",
    "em2g_ens_create", "em2g_ens_destroy", "em2g_ens_num_runs", "em2g_ens_set_stream",
    "em2g_ens_set_graph", "em2g_ens_set_fused", "em2g_ens_get_phase_ns",
    "em2g_ens_num_variants", "em2g_ens_set_variant",
    "em2g_ens_set_sort_interval", "em2g_ens_set_fields", "em2g_ens_get_fields",
    "em2g_ens_set_particles", "em2g_ens_set_particles_device", "em2g_ens_get_particles",
    "em2g_ens_step", "em2g_ens_get_step", "em2g_ens_diagnostics", "em2g_ens_get_counters",
]


class Em2gParams(C.Structure):
    """Mirror of struct em2g_params."""
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nsp", C.c_int32), ("isav", C.c_int32),
        ("precision", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("dt", C.c_double), ("c", C.c_double),
        ("qm", C.c_double * MAX_SPECIES), ("q", C.c_double * MAX_SPECIES),
        ("dn", C.c_double * MAX_SPECIES), ("am", C.c_double * MAX_SPECIES),
        ("tx", C.c_double * MAX_SPECIES), ("ty", C.c_double * MAX_SPECIES),
        ("np_max", C.c_int64 * MAX_SPECIES),
        ("cg_maxits", C.c_int32), ("energy_mode", C.c_int32),
        ("cg_eps", C.c_double), ("qme", C.c_double), ("wpe", C.c_double),
        ("device", C.c_int32), ("sort_interval", C.c_int32),
        ("smooth_current", C.c_int32), ("poisson", C.c_int32), ("staging_mib", C.c_int32),
        ("reserved", C.c_int32 * 13),
    ]


class Em2gError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"em2g status {status}: {msg}")
        self.status = status


_lib = None
_lib_checked = None


def lib() -> C.CDLL:
    """Load libem2g.so and declare argument types; raises if it is absent."""
    global _lib
    if _lib is None:
        _lib = _load(LIB_PATH)
    return _lib


def checked_lib() -> C.CDLL:
    """Load libem2g_checked.so, the bounds-checked build (its FP32 push counts
    and skips any out-of-range index instead of using it); raises if absent."""
    global _lib_checked
    if _lib_checked is None:
        _lib_checked = _load(LIB_CHECKED_PATH)
    return _lib_checked


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise RuntimeError(f"{path} not built: run `python -m maccpic_b200.build`")
    L = C.CDLL(path)
    dp, vp, ip, i64p = (C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_int),
                        C.POINTER(C.c_int64))
    pp = C.POINTER(Em2gParams)
    ctx = C.c_void_p
    sig = {
        "em2g_abi_version": (C.c_int, []),
        "em2g_last_error": (C.c_char_p, []),
        "em2g_params_init": (C.c_int, [pp]),
        "em2g_create": (C.c_int, [pp, C.POINTER(C.c_void_p)]),
        "em2g_destroy": (C.c_int, [ctx]),
        "em2g_set_stream": (C.c_int, [ctx, vp]),
        "em2g_synchronize": (C.c_int, [ctx]),
        "em2g_set_field": (C.c_int, [ctx, C.c_int, dp]),
        "em2g_get_field": (C.c_int, [ctx, C.c_int, dp]),
        "em2g_set_fields": (C.c_int, [ctx, dp]),
        "em2g_get_fields": (C.c_int, [ctx, dp]),
        "em2g_set_particles": (C.c_int, [ctx, C.c_int, C.c_int64] + [dp] * 6),
        "em2g_get_particles": (C.c_int, [ctx, C.c_int, i64p] + [dp] * 6),
        "em2g_particles_begin": (C.c_int, [ctx, C.c_int, C.c_int64]),
        "em2g_particles_add": (C.c_int, [ctx, C.c_int, C.c_int64, C.c_int64] + [vp] * 6
                               + [C.c_int]),
        "em2g_particles_end": (C.c_int, [ctx, C.c_int]),
        "em2g_get_particles_range": (C.c_int, [ctx, C.c_int, C.c_int64, C.c_int64] + [vp] * 6
                                     + [C.c_int]),
        "em2g_set_step": (C.c_int, [ctx, C.c_int]),
        "em2g_get_step": (C.c_int, [ctx, ip]),
        "em2g_set_fields_device": (C.c_int, [ctx, vp]),
        "em2g_get_fields_device": (C.c_int, [ctx, vp]),
        "em2g_field_device_ptr": (C.c_int, [ctx, C.c_int, C.POINTER(C.c_void_p)]),
        "em2g_move": (C.c_int, [ctx, dp]),
        "em2g_curnt": (C.c_int, [ctx]),
        "em2g_fields": (C.c_int, [ctx, C.c_int, dp, ip]),
        "em2g_smooth2": (C.c_int, [ctx, C.c_int]),
        "em2g_step": (C.c_int, [ctx, C.c_int, dp, dp, ip]),
        "em2g_set_particles_device": (C.c_int, [ctx, C.c_int, C.c_int64] + [vp] * 6),
        "em2g_move_curnt": (C.c_int, [ctx, dp]),
        "em2g_set_timing": (C.c_int, [ctx, C.c_int]),
        "em2g_get_counters": (C.c_int, [ctx, i64p, i64p, dp]),
        "em2g_reset_counters": (C.c_int, [ctx]),
        "em2g_smooth2_static": (C.c_int, [C.c_int, C.c_int, vp, vp]),
        "em2g_setv_device": (C.c_int, [C.POINTER(Em2gParams), C.c_int, vp, vp, C.c_int64, vp]),
        "em2g_diagnostics": (C.c_int, [ctx, dp, C.c_int]),
        "em2g_num_variants": (C.c_int, [ctx, ip]),
        "em2g_set_variant": (C.c_int, [ctx, C.c_int]),
        "em2g_get_variant": (C.c_int, [ctx, ip, C.c_char_p, C.c_int]),
        "em2g_set_sort_interval": (C.c_int, [ctx, C.c_int]),
        "em2g_set_stencils": (C.c_int, [ctx, C.c_int]),
        "em2g_get_stencils": (C.c_int, [ctx, C.POINTER(C.c_int)]),
        "em2g_selftest_waits": (C.c_int, [ctx, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "em2g_adj_create": (C.c_int, [ctx, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
        "em2g_adj_destroy": (C.c_int, [ctx]),
        "em2g_adj_forward": (C.c_int, [ctx, C.c_int]),
        "em2g_adj_keep_all_fields": (C.c_int, [ctx, C.c_int]),
        "em2g_adj_field_slots": (C.c_int, [ctx, C.c_int]),
        "em2g_adj_get_field_slots": (C.c_int, [ctx, C.POINTER(C.c_int)]),
        "em2g_adj_seed_fields_device": (C.c_int, [ctx, vp]),
        "em2g_adj_backward": (C.c_int, [ctx]),
        "em2g_adj_get_fields_device": (C.c_int, [ctx, vp]),
        "em2g_adj_get_particles_device": (C.c_int, [ctx, C.c_int] + [vp] * 5),
        "em2g_adj_get_initial_particles_device": (C.c_int, [ctx, C.c_int] + [vp] * 5),
        "em2g_ens_create": (C.c_int, [pp, C.c_int, C.POINTER(C.c_void_p)]),
        "em2g_ens_destroy": (C.c_int, [ctx]),
        "em2g_ens_num_runs": (C.c_int, [ctx, ip]),
        "em2g_ens_set_stream": (C.c_int, [ctx, vp]),
        "em2g_ens_set_graph": (C.c_int, [ctx, C.c_int]),
        "em2g_ens_set_fused": (C.c_int, [ctx, C.c_int]),
        "em2g_ens_get_phase_ns": (C.c_int, [ctx, i64p, C.c_int]),
        "em2g_ens_num_variants": (C.c_int, [ctx, ip]),
        "em2g_ens_set_variant": (C.c_int, [ctx, C.c_int]),
        "em2g_ens_set_sort_interval": (C.c_int, [ctx, C.c_int]),
        "em2g_ens_set_fields": (C.c_int, [ctx, C.c_int, dp]),
        "em2g_ens_get_fields": (C.c_int, [ctx, C.c_int, dp]),
        "em2g_ens_set_particles": (C.c_int, [ctx, C.c_int, C.c_int, C.c_int64] + [dp] * 6),
        "em2g_ens_set_particles_device": (C.c_int, [ctx, C.c_int, C.c_int, C.c_int64] + [vp] * 6),
        "em2g_ens_get_particles": (C.c_int, [ctx, C.c_int, C.c_int, i64p] + [dp] * 6),
        "em2g_ens_step": (C.c_int, [ctx, C.c_int, dp, dp, ip]),
        "em2g_ens_get_step": (C.c_int, [ctx, ip]),
        "em2g_ens_diagnostics": (C.c_int, [ctx, C.c_int, dp, C.c_int]),
        "em2g_ens_get_counters": (C.c_int, [ctx, i64p, i64p, i64p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def check(status: int, library: C.CDLL | None = None) -> None:
    """Raise Em2gError for a nonzero status, with the message of the library
    that returned it (libem2g.so unless another is given)."""
    if status != OK:
        raise Em2gError(status, (library or lib()).em2g_last_error().decode())
