"""em2's particle decomposition over GPUs.

em2 runs one MPI rank per core (pic/main.f90:19-20): every rank holds the
whole field grid and its own slice of each species; after ``curnt`` the
charge and current arrays are summed over ranks with MPI_ALLREDUCE
(pic/curnt.f90:363-376), the kinetic energies likewise
(pic/move.f90:214), and every rank then advances the identical fields
itself.  Here one process drives one GPU; the sums are
``torch.distributed.all_reduce`` (NCCL between GPUs, gloo for the CPU test
of the same orchestration), issued on the stream the library runs on.

:class:`ParticleDecomposition` is written against a small backend
interface so that the same code drives the GPU library (:class:`GpuBackend`)
and, in tests, the CPU oracle:

    backend.move_curnt() -> ake (nsp FP64 values of this rank's particles)
    backend.deposits()   -> list of tensor views of this rank's rho/J arrays
                            that hold deposits (each reduced in place)
    backend.fields(it)   -> (cg iterations, energies or None)
"""
from __future__ import annotations

import ctypes as C

import numpy as np


def rank_slice(n: int, rank: int, world: int) -> slice:
    """Contiguous share of n slots for `rank`, as em2 gives each rank
    MYRANK*maxnp+1 .. MYRANK*maxnp+np (pic/init.f90:25)."""
    lo = n * rank // world
    hi = n * (rank + 1) // world
    return slice(lo, hi)


class _DeviceArray:
    """__cuda_array_interface__ over library-owned device memory."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3}


class GpuBackend:
    """An :class:`~maccpic_b200.em2.Em2Gpu` context holding this rank's
    particles; the library runs on torch's current stream so that the
    collectives are ordered after its kernels.

    The fused push (em2g_move_curnt) deposits the whole current, jm + jp,
    into jxm, jym and jzm and leaves jxp, jyp and jzp zero (their only
    consumer is the sum, pic/fields.f90:211-214), so the arrays to sum over
    ranks are rho, jxm, jym and jzm: 4 of em2's 7 (pic/curnt.f90:363-369).
    rho and jxm are adjacent in the field block, so they go as one view."""

    def __init__(self, gpu):
        import torch
        from . import _lib
        self.g = gpu
        self.g.set_stream(torch.cuda.current_stream())
        ptr = C.c_void_p()
        _lib.check(gpu._L.em2g_field_device_ptr(gpu._h, _lib.FIELD_ID["rho"], C.byref(ptr)))
        w = (gpu.p.nx + 3) * (gpu.p.ny + 3)
        fp32 = gpu.p.precision == _lib.FP32
        typestr, word = ("<f4", 4) if fp32 else ("<f8", 8)
        base = ptr.value  # rho; then jxm, jxp, jym, jyp, jzm, jzp, each w words

        def view(first, count):
            return torch.as_tensor(_DeviceArray(base + first * w * word, count * w, typestr),
                                   device="cuda")
        self._views = [view(0, 2), view(3, 1), view(5, 1)]  # rho+jxm, jym, jzm

    def move_curnt(self):
        return self.g.move_curnt()

    def deposits(self):
        return self._views

    def fields(self, it):
        return self.g.fields(it)


class ParticleDecomposition:
    """One em2 main-loop pass per :meth:`step`, with rho/J and ake summed
    over the ranks of ``group`` between curnt and fields."""

    def __init__(self, backend, group=None):
        self.b = backend
        self.group = group

    def step(self, it: int) -> dict:
        import torch
        import torch.distributed as dist
        ake = np.asarray(self.b.move_curnt(), dtype=np.float64)
        if dist.is_initialized():
            deps = self.b.deposits()
            for d in deps:
                dist.all_reduce(d, op=dist.ReduceOp.SUM, group=self.group)
            t = torch.tensor(ake, dtype=torch.float64, device=deps[0].device)
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
            ake = t.cpu().numpy()
        n, e = self.b.fields(it)
        return {"ake": ake, "cg_iters": n, "energies": e}
