"""CPU oracle for the em2 time step -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package; it is the checker, never the product.  It wraps
``oracle/_build/libem2oracle.so``, a C restatement (FP64, serial, the
reference's evaluation order) of em2's move / curnt / fields / smooth2 /
Poisson / cgm (fanyumeng666/maccpic, pic/move.f90, pic/curnt.f90,
pic/fields.f90, pic/smooth.f90) plus its start-up (pic/init.f90,
pic/creator.f90, pic/smear.f90, pic/dran2.f90, pic/setv.f90) used to pin
the oracle against the reference's published initial-state numbers
(pic/RECONNECTION_MODEL.md:454-460).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libem2oracle.so")

NFIELD = 13
EX, EY, EZ, BX, BY, BZ, RHO, JXM, JXP, JYM, JYP, JZM, JZP = range(13)
FIELD_NAMES = ["ex", "ey", "ez", "bx", "by", "bz", "rho",
               "jxm", "jxp", "jym", "jyp", "jzm", "jzp"]


class _Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nsp", C.c_int32), ("isav", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("dt", C.c_double), ("c", C.c_double),
        ("qm", C.c_double * 4), ("q", C.c_double * 4), ("dn", C.c_double * 4),
        ("am", C.c_double * 4), ("tx", C.c_double * 4), ("ty", C.c_double * 4),
        ("cg_maxits", C.c_int32), ("energy_mode", C.c_int32),
        ("cg_eps", C.c_double), ("qme", C.c_double), ("wpe", C.c_double),
        ("smooth_current", C.c_int32),
    ]


class _LoadParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("npcel", C.c_int32), ("nsp", C.c_int32),
        ("nproc", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("dt", C.c_double), ("c", C.c_double),
        ("wce0", C.c_double), ("rmass", C.c_double), ("csw", C.c_double),
        ("csden", C.c_double), ("rtemp", C.c_double),
        ("temp", C.c_double * 2), ("aist", C.c_double * 2),
    ]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    srcs = [os.path.join(HERE, f) for f in
            ("em2_oracle.c", "em2_oracle.h", "em2_loader_oracle.c", "Makefile")]
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= max(os.path.getmtime(s) for s in srcs)):
        return LIB_PATH
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(build())
        dp, i64p = C.POINTER(C.c_double), C.POINTER(C.c_int64)
        pp = C.POINTER(_Params)
        L.em2o_move.restype = C.c_double
        L.em2o_move.argtypes = [pp, dp, C.c_int, C.c_int64, dp]
        L.em2o_curnt.restype = None
        L.em2o_curnt.argtypes = [pp, dp, C.c_int, C.c_int64, dp]
        for fn in ("em2o_fold", "em2o_yee"):
            getattr(L, fn).restype = None
            getattr(L, fn).argtypes = [pp, dp]
        L.em2o_smooth2.restype = None
        L.em2o_smooth2.argtypes = [pp, dp]
        L.em2o_poisson.restype = C.c_int
        L.em2o_poisson.argtypes = [pp, dp]
        L.em2o_energies.restype = None
        L.em2o_energies.argtypes = [pp, dp, dp]
        L.em2o_fields.restype = C.c_int
        L.em2o_fields.argtypes = [pp, dp, C.c_int, dp]
        L.em2o_step.restype = C.c_int
        L.em2o_step.argtypes = [pp, dp, C.c_int, i64p, C.POINTER(dp), dp, dp]
        L.em2o_step_mt.restype = C.c_int
        L.em2o_step_mt.argtypes = [pp, dp, C.c_int, i64p, C.POINTER(dp), dp, dp, C.c_int]
        lp = C.POINTER(_LoadParams)
        L.em2o_maxnp.restype = C.c_int64
        L.em2o_maxnp.argtypes = [lp]
        L.em2o_com_den.restype = None
        L.em2o_com_den.argtypes = [lp, dp, dp, dp, dp]
        L.em2o_init_fields.restype = None
        L.em2o_init_fields.argtypes = [lp, dp]
        L.em2o_creator.restype = C.c_int
        L.em2o_creator.argtypes = [lp, C.c_int, C.c_int64, C.POINTER(dp)]
        L.em2o_last_cg_residuals.restype = None
        L.em2o_last_cg_residuals.argtypes = [dp]
        L.em2o_setv.restype = None
        L.em2o_setv.argtypes = [pp, dp, C.c_int, C.c_int64, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class Params:
    """Run constants of one em2 configuration (pic/input.f90, pic/global.f90)."""
    nx: int
    ny: int
    dx: float
    dy: float
    dt: float
    qm: list
    q: list
    dn: list
    am: list
    nsp: int = 2
    isav: int = 20
    c: float = 1.0
    tx: list = field(default_factory=lambda: [0.0] * 4)
    ty: list = field(default_factory=lambda: [0.0] * 4)
    cg_maxits: int = 10000
    cg_eps: float = 1e-9
    energy_mode: int = 0
    qme: float = -1.0
    wpe: float = 1.0
    smooth_current: int = 0

    def ctype(self) -> _Params:
        P = _Params()
        P.nx, P.ny, P.nsp, P.isav = self.nx, self.ny, self.nsp, self.isav
        P.dx, P.dy, P.dt, P.c = self.dx, self.dy, self.dt, self.c
        for name in ("qm", "q", "dn", "am", "tx", "ty"):
            arr = getattr(P, name)
            vals = list(getattr(self, name)) + [0.0] * 4
            for i in range(4):
                arr[i] = float(vals[i])
        P.cg_maxits, P.energy_mode = self.cg_maxits, self.energy_mode
        P.cg_eps, P.qme, P.wpe = self.cg_eps, self.qme, self.wpe
        P.smooth_current = self.smooth_current
        return P

    @property
    def shape(self):
        return (self.ny + 3, self.nx + 3)


class State:
    """Field block (13, ny+3, nx+3) and per-species (6, n) particle blocks."""

    def __init__(self, params: Params, fields: np.ndarray, parts: list):
        self.p = params
        self._cp = params.ctype()
        self.fld = np.ascontiguousarray(fields, dtype=np.float64).copy()
        assert self.fld.shape == (NFIELD,) + params.shape
        self.parts = [np.ascontiguousarray(a, dtype=np.float64).copy() for a in parts]
        self.it = 0

    def copy(self) -> "State":
        s = State(self.p, self.fld, self.parts)
        s.it = self.it
        return s

    def move(self):
        L = lib()
        return [L.em2o_move(C.byref(self._cp), _dp(self.fld), isp,
                            self.parts[isp].shape[1], _dp(self.parts[isp]))
                for isp in range(self.p.nsp)]

    def curnt(self):
        L = lib()
        for isp in range(self.p.nsp):
            L.em2o_curnt(C.byref(self._cp), _dp(self.fld), isp,
                         self.parts[isp].shape[1], _dp(self.parts[isp]))

    def fields(self, it: int):
        e6 = np.full(6, np.nan)
        n = lib().em2o_fields(C.byref(self._cp), _dp(self.fld), it, _dp(e6))
        return n, e6

    def step(self, nthreads: int = 0):
        """One main-loop pass: move, curnt, it+=1, fields(it)."""
        L = lib()
        nsp = self.p.nsp
        ns = (C.c_int64 * nsp)(*[a.shape[1] for a in self.parts])
        ptrs = (C.POINTER(C.c_double) * nsp)(*[_dp(a) for a in self.parts])
        ake = np.zeros(4)
        e6 = np.full(6, np.nan)
        if nthreads:
            n = L.em2o_step_mt(C.byref(self._cp), _dp(self.fld), self.it, ns, ptrs,
                                _dp(ake), _dp(e6), nthreads)
        else:
            n = L.em2o_step(C.byref(self._cp), _dp(self.fld), self.it, ns, ptrs,
                            _dp(ake), _dp(e6))
        self.it += 1
        return {"cg_iters": n, "ake": ake[:nsp].copy(), "energies": e6}


def last_cg_residuals() -> np.ndarray:
    """Mean r^2 of the last cgm solve (any State or poisson call of this
    process): before the first iteration and at exit."""
    out = np.zeros(2)
    lib().em2o_last_cg_residuals(_dp(out))
    return out


def smooth2(params: Params, a: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.float64).copy()
    lib().em2o_smooth2(C.byref(params.ctype()), _dp(out))
    return out


def fold(params: Params, fld: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(fld, dtype=np.float64).copy()
    lib().em2o_fold(C.byref(params.ctype()), _dp(out))
    return out


def yee(params: Params, fld: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(fld, dtype=np.float64).copy()
    lib().em2o_yee(C.byref(params.ctype()), _dp(out))
    return out


def poisson(params: Params, fld: np.ndarray):
    out = np.ascontiguousarray(fld, dtype=np.float64).copy()
    n = lib().em2o_poisson(C.byref(params.ctype()), _dp(out))
    return out, n


def energies(params: Params, fld: np.ndarray) -> np.ndarray:
    e6 = np.zeros(6)
    f = np.ascontiguousarray(fld, dtype=np.float64)
    lib().em2o_energies(C.byref(params.ctype()), _dp(f), _dp(e6))
    return e6


# ---------------------------------------------------------------------------
# em2 start-up restated (pic/init.f90, pic/creator.f90, pic/smear.f90,
# pic/dran2.f90, pic/setv.f90), used to pin the oracle.
# ---------------------------------------------------------------------------
@dataclass
class Em2Setup:
    """Compile-time parameters of em2 (pic/input.f90:9-56) for the loader."""
    nx: int = 1024
    ny: int = 512
    npcel: int = 50
    nproc: int = 4
    dx: float = 0.1118
    wce0: float = -1.498147003616
    rmass: float = 100.0
    csw: float = 2.23606797749979
    csden: float = 5.0
    rtemp: float = 4.0
    temp: tuple = (4.4888888888e-02, 1.7955555555e-01 / 100.0)
    aist: tuple = (0.0, 0.0)
    isav: int = 20

    @property
    def dt(self):
        return self.dx * 0.7

    def ctype(self) -> _LoadParams:
        P = _LoadParams()
        P.nx, P.ny, P.npcel, P.nsp, P.nproc = self.nx, self.ny, self.npcel, 2, self.nproc
        P.dx, P.dy, P.dt, P.c = self.dx, self.dx, self.dt, 1.0
        P.wce0, P.rmass, P.csw, P.csden, P.rtemp = (self.wce0, self.rmass, self.csw,
                                                     self.csden, self.rtemp)
        P.temp[0], P.temp[1] = self.temp
        P.aist[0], P.aist[1] = self.aist
        return P


def setv(params: Params, fld: np.ndarray, isp: int, part: np.ndarray) -> np.ndarray:
    """em2's start-up push (pic/setv.f90:36-128) on a copy of one species'
    (6, n) block: v at t = 0 in, v and gamma at t = -dt/2 out."""
    out = np.ascontiguousarray(part, dtype=np.float64).copy()
    f = np.ascontiguousarray(fld, dtype=np.float64)
    lib().em2o_setv(C.byref(params.ctype()), _dp(f), int(isp), out.shape[1], _dp(out))
    return out


def em2_startup(setup: Em2Setup):
    """Run em2's fresh-run start-up (init -> creator -> setv) for every rank
    and return (Params, State, maxnp).  Species blocks hold rank 0's slots,
    then rank 1's, ... (the order of MYRANK*maxnp+j)."""
    L = lib()
    lp = setup.ctype()
    maxnp = int(L.em2o_maxnp(C.byref(lp)))
    q, qm, dn, am = (np.zeros(2) for _ in range(4))
    L.em2o_com_den(C.byref(lp), _dp(q), _dp(qm), _dp(dn), _dp(am))
    params = Params(nx=setup.nx, ny=setup.ny, dx=setup.dx, dy=setup.dx, dt=setup.dt,
                    qm=list(qm), q=list(q), dn=list(dn), am=list(am), isav=setup.isav)
    fld = np.zeros((NFIELD,) + params.shape)
    L.em2o_init_fields(C.byref(lp), _dp(fld))
    parts = [np.zeros((6, maxnp * setup.nproc)) for _ in range(2)]
    for rank in range(setup.nproc):
        blk = [np.zeros((6, maxnp)) for _ in range(2)]
        ptrs = (C.POINTER(C.c_double) * 2)(*[_dp(b) for b in blk])
        if L.em2o_creator(C.byref(lp), rank, maxnp, ptrs) != 0:
            raise RuntimeError("creator stopped (CDF inversion ran off the table)")
        for s in range(2):
            parts[s][:, rank * maxnp:(rank + 1) * maxnp] = blk[s]
    cp = params.ctype()
    for s in range(2):
        L.em2o_setv(C.byref(cp), _dp(fld), s, parts[s].shape[1], _dp(parts[s]))
    return params, State(params, fld, parts), maxnp
