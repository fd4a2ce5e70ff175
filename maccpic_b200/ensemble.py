"""Ensembles: many independent em2 runs advanced together on one GPU.

:class:`Em2Ensemble` owns one ``em2g_ens`` of the C ABI (include/em2g.h):
up to 128 FP32 runs, each with its own grid, species constants and
particles, stepped as :meth:`maccpic_b200.em2.Em2Gpu.step` steps one run,
but all of them per step in one captured CUDA graph -- one persistent push
launch for every run's particles and one launch per field stage for every
run's grid.  em2 itself runs one configuration per MPI job (pic/main.f90);
an ensemble is the same step for a batch of configurations.

:func:`harris_ensemble` draws the uneven double-Harris batch: grids
log-uniform from 128x64 to 1024x512, 16 to 64 particles per cell per
species, ion/electron mass ratio 25, 49 or 100, and a per-run seed and
flux-perturbation amplitude.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import NFIELD, check
from .em2 import RunParams, _check_out, _dp, stream_handle


class Em2Ensemble:
    """Independent FP32 runs resident on one GPU, stepped together."""

    def __init__(self, runs: list[RunParams], library=None):
        """`library`: the loaded C library to run on (default libem2g.so;
        _lib.checked_lib() is its bounds-checked build)."""
        self.runs = list(runs)
        self._L = library or _lib.lib()
        arr = (_lib.Em2gParams * len(self.runs))()
        for k, rp in enumerate(self.runs):
            if rp.precision != _lib.FP32:
                raise ValueError("ensemble runs are FP32 (RunParams.precision = FP32)")
            arr[k] = rp.ctype()
        self._arr = arr
        h = C.c_void_p()
        self._check(self._L.em2g_ens_create(arr, len(self.runs), C.byref(h)))
        self._h = h

    def _check(self, status: int) -> None:
        check(status, self._L)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._check(self._L.em2g_ens_destroy(self._h))
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

    def __len__(self):
        return len(self.runs)

    # ---- state copies ---------------------------------------------------
    def set_fields(self, run: int, fld: np.ndarray) -> None:
        a = np.ascontiguousarray(fld, dtype=np.float64)
        if a.shape != (NFIELD,) + self.runs[run].shape:
            raise ValueError(f"fields must have shape {(NFIELD,) + self.runs[run].shape}")
        self._check(self._L.em2g_ens_set_fields(self._h, run, _dp(a)))

    def get_fields(self, run: int, out: np.ndarray | None = None) -> np.ndarray:
        """Run `run`'s 13 arrays; into `out` (C-contiguous float64 of shape
        (13, ny+3, nx+3), e.g. pinned memory the caller keeps) if given."""
        shape = (NFIELD,) + self.runs[run].shape
        if out is None:
            out = np.empty(shape)
        else:
            _check_out(out, shape)
        self._check(self._L.em2g_ens_get_fields(self._h, run, _dp(out)))
        return out

    def set_particles(self, run: int, isp: int, part: np.ndarray) -> None:
        """part: (6, n) = x, y, vx, vy, vz, gamma; n must equal np_max[isp]."""
        a = np.ascontiguousarray(part, dtype=np.float64)
        if a.ndim != 2 or a.shape[0] != 6:
            raise ValueError("particles must have shape (6, n)")
        self._check(self._L.em2g_ens_set_particles(self._h, run, isp, a.shape[1],
                                             *[_dp(a[k]) for k in range(6)]))

    def set_particles_device(self, run: int, isp: int, part) -> None:
        """part: a CUDA float64 tensor (6, n) on the ensemble's device."""
        import torch
        if part.dtype != torch.float64 or part.dim() != 2 or part.shape[0] != 6:
            raise ValueError("particles must be a float64 tensor of shape (6, n)")
        part = part.contiguous()
        torch.cuda.current_stream(part.device).synchronize()
        ptrs = [C.c_void_p(part[k].data_ptr()) for k in range(6)]
        self._check(self._L.em2g_ens_set_particles_device(self._h, run, isp, part.shape[1], *ptrs))

    def get_particles(self, run: int, isp: int, out: np.ndarray | None = None) -> np.ndarray:
        """(6, n) = x, y, vx, vy, vz, gamma of run `run`, species `isp`, in
        slot order; into `out` (C-contiguous float64 of that shape) if given."""
        n = C.c_int64()
        self._check(self._L.em2g_ens_get_particles(self._h, run, isp, C.byref(n),
                                             *([None] * 6)))
        if out is None:
            out = np.empty((6, n.value))
        else:
            _check_out(out, (6, n.value))
        self._check(self._L.em2g_ens_get_particles(self._h, run, isp, C.byref(n),
                                             *[_dp(out[k]) for k in range(6)]))
        return out

    # ---- stepping ---------------------------------------------------------
    def step(self, nsteps: int = 1) -> dict:
        """nsteps of every run.  ake (nruns, 4), energies (nruns, 6) of the
        runs whose isav divides the step count (NaN rows otherwise),
        cg_iters (nruns,) of the last step."""
        nr = len(self.runs)
        ake = np.zeros((nr, 4))
        e6 = np.full((nr, 6), np.nan)
        it = (C.c_int * nr)()
        self._check(self._L.em2g_ens_step(self._h, int(nsteps), _dp(ake), _dp(e6), it))
        return {"ake": ake, "energies": e6, "cg_iters": np.array(it[:], dtype=np.int64)}

    @property
    def it(self) -> int:
        v = C.c_int()
        self._check(self._L.em2g_ens_get_step(self._h, C.byref(v)))
        return v.value

    def set_graph(self, on: bool) -> None:
        self._check(self._L.em2g_ens_set_graph(self._h, 1 if on else 0))

    def phase_ms(self, n: int = 24):
        """Durations (ms) of the last fused step's phases: from the launch's
        start to its first grid barrier, then between barriers."""
        out = (C.c_int64 * n)()
        self._check(self._L.em2g_ens_get_phase_ns(self._h, out, n))
        return [v / 1e6 for v in out]

    def set_fused(self, on: bool) -> None:
        """True: each step is one persistent, cooperative kernel launch
        (em2g_ens_set_fused); False: one launch per stage."""
        self._check(self._L.em2g_ens_set_fused(self._h, 1 if on else 0))

    def num_variants(self) -> int:
        n = C.c_int()
        self._check(self._L.em2g_ens_num_variants(self._h, C.byref(n)))
        return n.value

    def set_variant(self, v: int) -> None:
        self._check(self._L.em2g_ens_set_variant(self._h, int(v)))

    def set_sort_interval(self, k: int) -> None:
        """Regroup every run's particles by cell on every k-th step and update
        them in place in between (k * c * dt < dx, dy in every run)."""
        self._check(self._L.em2g_ens_set_sort_interval(self._h, int(k)))
        for r in self.runs:
            r.sort_interval = int(k)

    def max_sort_interval(self) -> int:
        """The largest interval the drift bound allows in every run."""
        import math
        k = min(math.ceil(min(r.dx, r.dy) / (r.c * r.dt)) - 1 for r in self.runs)
        return max(1, k)

    def set_stream(self, stream) -> None:
        """As Em2Gpu.set_stream."""
        self._check(self._L.em2g_ens_set_stream(self._h, stream_handle(stream)))

    def counters(self) -> dict:
        k, g, per = C.c_int64(), C.c_int64(), C.c_int64()
        self._check(self._L.em2g_ens_get_counters(self._h, C.byref(k), C.byref(g), C.byref(per)))
        return {"kernel_launches": k.value, "graph_launches": g.value,
                "kernels_per_step": per.value}

    def diagnostics(self, run: int) -> dict:
        out = np.full(10, np.nan)
        self._check(self._L.em2g_ens_diagnostics(self._h, run, _dp(out), 10))
        return {"energies": out[:6].copy(), "flux": out[6:8].copy(),
                "poisson_r2": out[8:10].copy()}

    @property
    def particles(self) -> int:
        return int(sum(sum(rp.np_max[: rp.nsp]) for rp in self.runs))


def harris_ensemble(nruns: int = 64, seed: int = 0, lo=(128, 64), hi=(1024, 512),
                    ppc=(16, 64), mass_ratios=(25.0, 49.0, 100.0), steps: int = 500):
    """The uneven batch of double-Harris runs: per run a grid log-uniform in
    area between lo and hi (aspect 2:1, nx a multiple of 16), particles per
    cell uniform in ppc, a mass ratio from mass_ratios, a flux perturbation
    psi0 uniform in [0.05, 0.15] B0 d_i and its own seed."""
    from .loader import HarrisConfig
    rng = np.random.Generator(np.random.Philox(key=[seed, 0xE45]))
    out = []
    for k in range(nruns):
        nx = math.exp(rng.uniform(math.log(lo[0]), math.log(hi[0])))
        nx = int(min(hi[0], max(lo[0], 16 * round(nx / 16))))
        out.append(HarrisConfig(nx=nx, ny=nx // 2, ppc=int(rng.integers(ppc[0], ppc[1] + 1)),
                                mass_ratio=float(rng.choice(mass_ratios)),
                                psi0_over_b0di=float(rng.uniform(0.05, 0.15)),
                                steps=steps, seed=int(rng.integers(1 << 30))))
    return out


def load_harris(cfgs, device="cuda") -> Em2Ensemble:
    """An ensemble holding the initial double-Harris state of each config,
    particles sampled on the GPU."""
    from .loader import initial_fields, sample_particles_torch
    runs = []
    for c in cfgs:
        n = c.nx * c.ny * c.ppc
        runs.append(c.run_params(np_max=[n, n], precision=_lib.FP32))
    ens = Em2Ensemble(runs)
    try:
        for r, c in enumerate(cfgs):
            ens.set_fields(r, initial_fields(c))
            for s, part in enumerate(sample_particles_torch(c, device=device)):
                ens.set_particles_device(r, s, part)
                del part
    except Exception:
        ens.close()
        raise
    return ens
