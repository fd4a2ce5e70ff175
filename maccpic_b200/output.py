"""em2's diagnostic files, written from the GPU state by a background thread.

The quantities are computed on the GPU (energies by ``em2g_fields`` /
``em2g_diagnostics`` in FP64, the arrays by one device-to-host copy each);
the host formatting and file writes run on a worker thread so the time
loop does not wait for them.  Formats follow em2's ``output``
(pic/output.f90):

* ``ene###.hst``     one line per call: time, exe, eye, eze, bxe, bye, bze,
                     ake(1:nsp)/anme, total, Fortran format (11e13.5)
                     (pic/output.f90:191-199)
* ``cf-p1_###.bin``  Bz frames every 100 steps, raw (0:nx+2,0:ny+2) REAL(8),
                     frame it/100 at byte (frame mod 30)*size*8 of file
                     it/100/30 + 1 (pic/output.f90:151-169)
* ``ex_TTTTT.dat``.. 2D snapshots, ny lines of nx values (1024e13.5)
                     (pic/output.f90:89-142)
* ``ex###.hst`` ..   the profile along y at ix = nx/2, one line per call
                     (pic/output.f90:242-247)
"""
from __future__ import annotations

import math
import os
import queue
import threading

import numpy as np

FIELDS6 = ["ex", "ey", "ez", "bx", "by", "bz"]


def fortran_e(v: float, w: int = 13, d: int = 5) -> str:
    """Fortran Ew.d edit descriptor as gfortran writes it: 0.ddddE+xx."""
    if v != v:
        return "NaN".rjust(w)
    if math.isinf(v):
        return ("-Infinity" if v < 0 else "Infinity").rjust(w)
    if v == 0.0:
        s = "0." + "0" * d + "E+00"
        return (("-" if math.copysign(1.0, v) < 0 else "") + s).rjust(w)
    a = abs(v)
    e = math.floor(math.log10(a)) + 1
    m = round(a / 10.0 ** e, d)
    if m >= 1.0:  # rounding carried into a new digit
        m /= 10.0
        e += 1
    if m < 0.1:
        m *= 10.0
        e -= 1
    digits = f"{m:.{d}f}"[2:]
    exp = f"E{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) < 100 else \
        f"{'+' if e >= 0 else '-'}{abs(e):03d}"
    s = ("-" if v < 0 else "") + "0." + digits + exp
    return s.rjust(w)


def fortran_row(values, w: int = 13, d: int = 5) -> str:
    return "".join(fortran_e(float(v), w, d) for v in values)


class Em2Output:
    """Writes em2's diagnostic files into `directory` on a worker thread."""

    def __init__(self, directory: str, nx: int, ny: int, dt: float, anme: float,
                 ifile: int = 1, frames_per_file: int = 30):
        self.dir = directory
        os.makedirs(directory, exist_ok=True)
        self.nx, self.ny, self.dt, self.anme = nx, ny, dt, anme
        self.ifile = ifile
        self.fpf = frames_per_file
        self._q: queue.Queue = queue.Queue(maxsize=8)
        self._err = None
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        while True:
            job = self._q.get()
            if job is None:
                return
            try:
                job()
            except Exception as e:  # reported by close()
                self._err = e

    def _submit(self, fn):
        if self._err is not None:
            raise RuntimeError("output writer failed") from self._err
        self._q.put(fn)

    def close(self):
        self._q.put(None)
        self._t.join()
        if self._err is not None:
            raise RuntimeError("output writer failed") from self._err

    # ---- em2's output call -----------------------------------------------------
    def output(self, run, it: int, ake, isav: int = 20, iphs: int = 1000):
        """What em2's ``output`` writes at step ``it`` (pic/output.f90:130-247),
        from a GPU run (:class:`~maccpic_b200.em2.Em2Gpu`): the energy line at
        it == 1 and every isav steps, with the field energies computed on the
        GPU in FP64 for the current fields (``em2g_diagnostics``); the Bz frame
        every 100 steps; the profiles every isav steps; the 2D snapshots every
        iphs steps.  Arrays are copied from the device here, and formatted and
        written on the worker thread."""
        fields = None
        if it == 1 or (it != 0 and it % isav == 0):
            self.energies(it, run.diagnostics()["energies"], ake)
            fields = run.get_fields()
            # a new profile file every idata = 1024 records (pic/output.f90:204-215)
            self.profiles(fields, iii=(it // isav) // 1024 + 1)
        if it % 100 == 0:
            self.bz_frame(it, run.get_field("bz"))
        if it % iphs == 0:
            self.snapshot(it, fields if fields is not None else run.get_fields())

    # ---- writers -----------------------------------------------------------
    def energies(self, it: int, e6, ake):
        """ene###.hst line (pic/output.f90:191-199); ake as move returns it."""
        e6 = [float(x) for x in e6]
        kin = [float(a) / self.anme for a in ake]
        total = sum(e6) + sum(kin)
        line = fortran_row([it * self.dt] + e6 + kin + [total]) + "\n"
        path = os.path.join(self.dir, f"ene{self.ifile:03d}.hst")

        def job():
            with open(path, "a") as f:
                f.write(line)
        self._submit(job)

    def bz_frame(self, it: int, bz: np.ndarray):
        """cf-p1 frame of step it (a multiple of 100), pic/output.f90:151-169."""
        if it % 100:
            raise ValueError("cf-p1 frames are written at multiples of 100 steps")
        frame = it // 100
        findex = frame // self.fpf + 1
        pos = (frame % self.fpf) * bz.size * 8
        data = np.ascontiguousarray(bz, dtype="<f8").tobytes()
        path = os.path.join(self.dir, f"cf-p1_{findex:03d}.bin")
        first = frame % self.fpf == 0

        def job():
            mode = "wb" if first or not os.path.exists(path) else "r+b"
            with open(path, mode) as f:
                f.seek(pos)
                f.write(data)
        self._submit(job)

    def snapshot(self, it: int, fields):
        """2D snapshots ex_TTTTT.dat ... (pic/output.f90:89-142); fields is the
        (13 or 6, ny+3, nx+3) block."""
        itime = int(it * self.dt)
        arrays = {n: np.array(fields[k][1:self.ny + 1, 1:self.nx + 1])
                  for k, n in enumerate(FIELDS6)}

        def job():
            for n, a in arrays.items():
                with open(os.path.join(self.dir, f"{n}_{itime:05d}.dat"), "w") as f:
                    for row in a:
                        for lo in range(0, row.size, 1024):
                            f.write(fortran_row(row[lo:lo + 1024]) + "\n")
        self._submit(job)

    def profiles(self, fields, iii: int = 1):
        """One line per component along y at ix = nx/2 (pic/output.f90:242-247)."""
        cols = {n: np.array(fields[k][1:self.ny + 1, self.nx // 2])
                for k, n in enumerate(FIELDS6)}

        def job():
            for n, col in cols.items():
                with open(os.path.join(self.dir, f"{n}{iii:03d}.hst"), "a") as f:
                    for lo in range(0, col.size, 1024):
                        f.write(fortran_row(col[lo:lo + 1024]) + "\n")
        self._submit(job)
