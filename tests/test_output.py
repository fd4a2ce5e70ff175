"""em2's diagnostic files (pic/output.f90): Fortran e13.5 formatting, the
energy history line, Bz frame placement and the 2D snapshot layout."""
import os

import numpy as np


def test_fortran_e13_5():
    from maccpic_b200.output import fortran_e
    assert fortran_e(1.0) == "  0.10000E+01"
    assert fortran_e(-0.0257) == " -0.25700E-01"
    assert fortran_e(0.0) == "  0.00000E+00"
    assert fortran_e(123456.7) == "  0.12346E+06"
    assert fortran_e(9.999996) == "  0.10000E+02"   # rounding carries a digit
    assert fortran_e(1.5e-120) == "  0.15000-119"   # three-digit exponent drops the E
    assert all(len(fortran_e(v)) == 13 for v in (1e-5, -3.3e7, 42.0))


def test_energy_line_and_frames(tmp_path):
    from maccpic_b200.output import Em2Output
    out = Em2Output(str(tmp_path), nx=8, ny=4, dt=0.05, anme=2.0)
    out.energies(20, [1, 2, 3, 4, 5, 6], [10.0, 20.0])
    bz = np.arange(11 * 7, dtype=float).reshape(7, 11)
    out.bz_frame(100, bz)       # frame 1 of file 001
    out.bz_frame(3100, bz * 2)  # frame 31 -> file 002, slot 1
    out.snapshot(1000, np.random.default_rng(0).normal(size=(13, 7, 11)))
    out.close()
    line = open(tmp_path / "ene001.hst").read()
    vals = [float(line[k:k + 13]) for k in range(0, len(line.rstrip()), 13)]
    # time, exe..bze, ake/anme for 2 species, total (10 of the 11 slots)
    np.testing.assert_allclose(vals, [1.0, 1, 2, 3, 4, 5, 6, 5.0, 10.0, 36.0], rtol=1e-5)
    f1 = (tmp_path / "cf-p1_001.bin").read_bytes()
    assert len(f1) == 2 * bz.size * 8
    np.testing.assert_array_equal(np.frombuffer(f1[bz.size * 8:], "<f8"), bz.ravel())
    f2 = (tmp_path / "cf-p1_002.bin").read_bytes()
    np.testing.assert_array_equal(np.frombuffer(f2[bz.size * 8:], "<f8"), 2 * bz.ravel())
    snap = open(tmp_path / "ex_00050.dat").read().splitlines()
    assert len(snap) == 4 and all(len(r) == 8 * 13 for r in snap)
