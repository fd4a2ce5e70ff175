"""Host-side mirror of em2's step interface on the GPU.

em2 (fanyumeng666/maccpic, pic/) advances its state with parameterless
subroutines acting on the module ``global`` (pic/global.f90:31-45):

    call move     ! pic/move.f90:2     -> Em2Gpu.move()   (returns ake)
    call curnt    ! pic/curnt.f90:2    -> Em2Gpu.curnt()
    it = it + 1
    call fields   ! pic/fields.f90:2   -> Em2Gpu.fields(it)
    call smooth2(sm)  ! pic/smooth.f90:95 -> Em2Gpu.smooth2(name)

:class:`Em2Gpu` owns one libem2g context; the state that ``global`` holds
lives on the GPU and is copied in and out with :meth:`set_fields`,
:meth:`get_fields`, :meth:`set_particles`, :meth:`get_particles`, in the
reference's layouts ((ny+3, nx+3) REAL(8) field arrays; x, y, vx, vy, vz,
gamma per species).  Errors raise :class:`~maccpic_b200._lib.Em2gError`,
where em2 itself would print and continue or stop.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import FIELD_ID, FIELD_NAMES, NFIELD, check


@dataclass
class RunParams:
    """Run constants: pic/input.f90:9-43 and derived pic/global.f90:18-28.

    Per-species values follow com_den (pic/input.f90:61-69) and init
    (pic/init.f90:116-119): ``qm`` charge/mass, ``q`` macro charge, ``dn``
    relative density, ``am`` macro mass."""
    nx: int
    ny: int
    dx: float
    dy: float
    dt: float
    qm: list
    q: list
    dn: list
    am: list
    np_max: list
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
    precision: int = _lib.FP64
    device: int = 0
    sort_interval: int = 0
    smooth_current: int = 0     # 1: smooth2 the current every step (not in em2)
    poisson: int = 0            # 0: em2's CG; 1: exact spectral solve (FP64, 2^k sides)
    staging_mib: int = 0        # device staging for particle copies (0: the default)

    @property
    def shape(self):
        return (self.ny + 3, self.nx + 3)

    def ctype(self) -> _lib.Em2gParams:
        P = _lib.Em2gParams()
        check(_lib.lib().em2g_params_init(C.byref(P)))
        for name in ("nx", "ny", "nsp", "isav", "precision", "dx", "dy", "dt", "c",
                     "cg_maxits", "energy_mode", "cg_eps", "qme", "wpe", "device",
                     "sort_interval", "smooth_current", "poisson", "staging_mib"):
            setattr(P, name, getattr(self, name))
        for name in ("qm", "q", "dn", "am", "tx", "ty"):
            arr = getattr(P, name)
            vals = list(getattr(self, name)) + [0.0] * 4
            for i in range(4):
                arr[i] = float(vals[i])
        vals = list(self.np_max) + [0] * 4
        for i in range(4):
            P.np_max[i] = int(vals[i])
        return P


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _check_out(out: np.ndarray, shape) -> None:
    """A caller's output buffer must be C-contiguous float64 of `shape`."""
    if (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.shape != tuple(shape)
            or not out.flags.c_contiguous or not out.flags.writeable):
        raise ValueError(f"out must be a writeable C-contiguous float64 array of shape "
                         f"{tuple(shape)}")


CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: the legacy default stream's handle


def stream_handle(stream) -> C.c_void_p:
    """The cudaStream_t to hand to the library: None -> NULL (the library's
    own stream); a torch stream or an int handle as is, except the default
    stream (handle 0, which the library would read as NULL) -> the legacy
    default stream's explicit handle."""
    if stream is None:
        return C.c_void_p(0)
    handle = getattr(stream, "cuda_stream", stream)
    return C.c_void_p(handle if handle else CUDA_STREAM_LEGACY)


class Em2Gpu:
    """One em2 run resident on one GPU."""

    def __init__(self, params: RunParams, library: C.CDLL | None = None):
        """`library`: the loaded C library to run on (default libem2g.so;
        _lib.checked_lib() is its bounds-checked build)."""
        self.p = params
        self._L = library or _lib.lib()
        self._P = params.ctype()
        h = C.c_void_p()
        self._check(self._L.em2g_create(C.byref(self._P), C.byref(h)))
        self._h = h

    def _check(self, status: int) -> None:
        check(status, self._L)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._check(self._L.em2g_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- state copies ---------------------------------------------------
    def set_fields(self, fld: np.ndarray) -> None:
        """All 13 arrays, shape (13, ny+3, nx+3), enum em2g_field order."""
        a = np.ascontiguousarray(fld, dtype=np.float64)
        if a.shape != (NFIELD,) + self.p.shape:
            raise ValueError(f"fields must have shape {(NFIELD,) + self.p.shape}")
        self._check(self._L.em2g_set_fields(self._h, _dp(a)))

    def get_fields(self, out: np.ndarray | None = None) -> np.ndarray:
        """All 13 arrays, shape (13, ny+3, nx+3); into `out` (C-contiguous
        float64 of that shape, e.g. pinned memory the caller keeps) if given."""
        shape = (NFIELD,) + self.p.shape
        if out is None:
            out = np.empty(shape)
        else:
            _check_out(out, shape)
        self._check(self._L.em2g_get_fields(self._h, _dp(out)))
        return out

    def set_field(self, name: str, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.p.shape:
            raise ValueError(f"field must have shape {self.p.shape}")
        self._check(self._L.em2g_set_field(self._h, FIELD_ID[name], _dp(a)))

    def get_field(self, name: str) -> np.ndarray:
        out = np.empty(self.p.shape)
        self._check(self._L.em2g_get_field(self._h, FIELD_ID[name], _dp(out)))
        return out

    def set_particles(self, isp: int, part: np.ndarray) -> None:
        """part: (6, n) = x, y, vx, vy, vz, gamma in slot order."""
        a = np.ascontiguousarray(part, dtype=np.float64)
        if a.ndim != 2 or a.shape[0] != 6:
            raise ValueError("particles must have shape (6, n)")
        n = a.shape[1]
        self._check(self._L.em2g_set_particles(self._h, isp, n, *[_dp(a[k]) for k in range(6)]))

    def set_particles_device(self, isp: int, part) -> None:
        """part: a CUDA tensor (6, n) float64 on this context's device; the
        library copies it on its stream (call set_stream first to order it
        after the producer)."""
        import torch
        if part.dtype != torch.float64 or part.dim() != 2 or part.shape[0] != 6:
            raise ValueError("particles must be a float64 tensor of shape (6, n)")
        part = part.contiguous()
        n = part.shape[1]
        ptrs = [C.c_void_p(part[k].data_ptr()) for k in range(6)]
        self._check(self._L.em2g_set_particles_device(self._h, isp, n, *ptrs))

    def set_particles_slices(self, isp: int, n: int, slices) -> None:
        """n particles of species isp handed over one slice at a time, for
        sets too large to hold whole (em2g_particles_begin / add / end):
        `slices` yields (6, m) float64 arrays -- numpy (host) or CUDA
        tensors on this context's device -- in slot order, m summing to n.
        The species keeps its old particles unless all n arrive and pass
        the library's checks."""
        L = self._L
        self._check(L.em2g_particles_begin(self._h, isp, int(n)))
        first = 0
        try:
            for a in slices:
                if isinstance(a, np.ndarray):
                    a = np.ascontiguousarray(a, dtype=np.float64)
                    ptrs = [C.c_void_p(a[k].ctypes.data) for k in range(6)]
                    dev = 0
                else:
                    import torch
                    if a.dtype != torch.float64 or not a.is_cuda:
                        raise ValueError("device slices must be float64 CUDA tensors")
                    a = a.contiguous()
                    ptrs = [C.c_void_p(a[k].data_ptr()) for k in range(6)]
                    dev = 1
                if a.ndim != 2 or a.shape[0] != 6:
                    raise ValueError("slices must have shape (6, m)")
                m = int(a.shape[1])
                self._check(L.em2g_particles_add(self._h, isp, first, m, *ptrs, dev))
                # the slice is read on the library's stream: wait for it before
                # the caller may free or reuse its memory
                self._check(L.em2g_synchronize(self._h))
                first += m
        finally:
            rc = L.em2g_particles_end(self._h, isp)
        self._check(rc)

    def get_particles_range(self, isp: int, first: int, count: int, out=None):
        """Slots first..first+count-1 of species isp as (6, count) x, y, vx,
        vy, vz, gamma: into `out` (a C-contiguous float64 numpy array, or a
        float64 CUDA tensor for a device-side copy) or a new numpy array."""
        if out is None:
            out = np.empty((6, count))
        if isinstance(out, np.ndarray):
            _check_out(out, (6, count))
            ptrs = [C.c_void_p(out[k].ctypes.data) for k in range(6)]
            dev = 0
        else:
            if tuple(out.shape) != (6, count) or not out.is_contiguous() or not out.is_cuda:
                raise ValueError("out must be a contiguous (6, count) float64 CUDA tensor")
            ptrs = [C.c_void_p(out[k].data_ptr()) for k in range(6)]
            dev = 1
        self._check(self._L.em2g_get_particles_range(self._h, isp, int(first), int(count), *ptrs, dev))
        return out

    def set_stream(self, stream) -> None:
        """Enqueue further work on this cudaStream_t (int handle, or a torch
        stream); None returns to the context's own stream."""
        self._check(self._L.em2g_set_stream(self._h, stream_handle(stream)))

    def num_variants(self) -> int:
        n = C.c_int()
        self._check(self._L.em2g_num_variants(self._h, C.byref(n)))
        return n.value

    def set_variant(self, v: int) -> None:
        self._check(self._L.em2g_set_variant(self._h, int(v)))

    def set_sort_interval(self, k: int) -> None:
        """Regroup particles by cell every k-th step (FP32; k*c*dt < dx, dy)."""
        self._check(self._L.em2g_set_sort_interval(self._h, int(k)))
        self.p.sort_interval = int(k)

    def set_stencils(self, mode: int) -> None:
        """How the Yee updates and smooth2 passes read their arrays: 0 direct
        loads per cell, 1 tiles staged in shared memory by tensor copies.
        The results are the same; only the speed differs."""
        self._check(self._L.em2g_set_stencils(self._h, int(mode)))

    def stencils(self) -> int:
        m = C.c_int(0)
        self._check(self._L.em2g_get_stencils(self._h, C.byref(m)))
        return m.value

    def max_sort_interval(self) -> int:
        """The largest interval the drift bound allows (1 for FP64)."""
        if self.p.precision != _lib.FP32:
            return 1
        import math
        step = self.p.c * self.p.dt / min(self.p.dx, self.p.dy)
        return max(1, math.ceil(1.0 / step) - 1)

    def variant(self):
        """(index, name) of the fast-push kernel variant in use."""
        v = C.c_int()
        buf = C.create_string_buffer(64)
        self._check(self._L.em2g_get_variant(self._h, C.byref(v), buf, 64))
        return v.value, buf.value.decode()

    def set_timing(self, on: bool) -> None:
        self._check(self._L.em2g_set_timing(self._h, int(bool(on))))

    def counters(self) -> dict:
        a, b, ms = C.c_int64(), C.c_int64(), C.c_double()
        self._check(self._L.em2g_get_counters(self._h, C.byref(a), C.byref(b), C.byref(ms)))
        return {"kernel_launches": a.value, "push_launches_timed": b.value,
                "push_ms": ms.value}

    def reset_counters(self) -> None:
        self._check(self._L.em2g_reset_counters(self._h))

    def get_particles(self, isp: int, out: np.ndarray | None = None) -> np.ndarray:
        """(6, n) = x, y, vx, vy, vz, gamma in slot order; into `out`
        (C-contiguous float64 of that shape) if given."""
        n = C.c_int64()
        self._check(self._L.em2g_get_particles(self._h, isp, C.byref(n), *([None] * 6)))
        if out is None:
            out = np.empty((6, n.value))
        else:
            _check_out(out, (6, n.value))
        if n.value:
            self._check(self._L.em2g_get_particles(self._h, isp, C.byref(n),
                                             *[_dp(out[k]) for k in range(6)]))
        return out

    @property
    def it(self) -> int:
        v = C.c_int()
        self._check(self._L.em2g_get_step(self._h, C.byref(v)))
        return v.value

    @it.setter
    def it(self, value: int) -> None:
        self._check(self._L.em2g_set_step(self._h, int(value)))

    # ---- the subroutines --------------------------------------------------
    def move(self) -> np.ndarray:
        """pic/move.f90: gather + Boris; returns ake(1:nsp)."""
        ake = np.zeros(4)
        self._check(self._L.em2g_move(self._h, _dp(ake)))
        return ake[: self.p.nsp]

    def move_curnt(self) -> np.ndarray:
        """move then curnt in one fused particle kernel; returns ake."""
        ake = np.zeros(4)
        self._check(self._L.em2g_move_curnt(self._h, _dp(ake)))
        return ake[: self.p.nsp]

    def curnt(self) -> None:
        """pic/curnt.f90: deposit jm, move + wrap, deposit rho and jp."""
        self._check(self._L.em2g_curnt(self._h))

    def fields(self, it: int):
        """pic/fields.f90 for step ``it``; returns (cg iterations, energies or None)."""
        e6 = np.full(6, np.nan)
        n = C.c_int()
        self._check(self._L.em2g_fields(self._h, int(it), _dp(e6), C.byref(n)))
        return n.value, (e6 if it % self.p.isav == 0 else None)

    def diagnostics(self) -> dict:
        """Field energies of the current fields, reconnected flux of both
        sheets and the last Poisson residuals (FP64, computed on the GPU)."""
        out = np.zeros(10)
        self._check(self._L.em2g_diagnostics(self._h, _dp(out), 10))
        return {"energies": out[:6].copy(), "flux": out[6:8].copy(),
                "poisson_r2_before": out[8], "poisson_r2_after": out[9]}

    def smooth2(self, name: str) -> None:
        """pic/smooth.f90:95 on one resident field array."""
        self._check(self._L.em2g_smooth2(self._h, FIELD_ID[name]))

    def step(self, nsteps: int = 1) -> dict:
        """nsteps of {move; curnt; it+=1; fields(it)} on the fused fast path."""
        ake = np.zeros(4)
        e6 = np.full(6, np.nan)
        n = C.c_int()
        self._check(self._L.em2g_step(self._h, int(nsteps), _dp(ake), _dp(e6), C.byref(n)))
        return {"ake": ake[: self.p.nsp].copy(), "cg_iters": n.value,
                "energies": e6 if self.it % self.p.isav == 0 else None}


def setv_device(params: RunParams, isp: int, fields, parts, stream=None) -> None:
    """em2's start-up push (pic/setv.f90:36-128) in place on the GPU: the
    velocities of ``parts`` -- a (6, n) float64 CUDA tensor (x, y, vx, vy,
    vz, gamma), v at t = 0 -- pushed back to t = -dt/2 with the E and B of
    ``fields`` (a (13, ny+3, nx+3) float64 CUDA tensor, em2's layout)
    gathered with linear weights, gamma recomputed.  Bitwise em2's
    arithmetic; particles outside the box or not slower than c raise
    :class:`~maccpic_b200._lib.Em2gError` and leave ``parts`` unchanged.
    Runs on ``stream`` (default: torch's current stream) and returns once
    the push is enqueued."""
    import torch
    shape = (NFIELD, params.ny + 3, params.nx + 3)
    for name, t, want in (("fields", fields, shape), ("parts", parts, None)):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64
                and t.is_contiguous()):
            raise ValueError(f"{name} must be a contiguous float64 CUDA tensor")
        if want is not None and tuple(t.shape) != want:
            raise ValueError(f"fields must have shape {want}")
    if parts.dim() != 2 or parts.shape[0] != 6:
        raise ValueError("parts must have shape (6, n)")
    if stream is None:
        stream = torch.cuda.current_stream(parts.device)
    p = params.ctype()
    with torch.cuda.device(parts.device):
        check(_lib.lib().em2g_setv_device(C.byref(p), int(isp), C.c_void_p(fields.data_ptr()),
                                          C.c_void_p(parts.data_ptr()), int(parts.shape[1]),
                                          stream_handle(stream)))
