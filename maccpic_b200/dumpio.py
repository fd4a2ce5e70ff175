"""em2's restart files, read and written from the GPU state.

At its last step em2 writes (pic/output.f90:279-364), and ``cont`` reads
back (pic/cont.f90:21-92), gfortran sequential unformatted files in which
every WRITE is one record framed by its byte length as a 4-byte integer
before and after the data:

  fld.fin            6 records of (nx+3)(ny+3) REAL(8): bx, by, bz, ex, ey, ez
  rhoj.fin           7 records: rho, jxm, jxp, jym, jyp, jzm, jzp
  x_rankNNN.fin ...  one 8-byte record per particle, species 1 first, slots
  (y, vx, vy, vz, g)  MYRANK*maxnp+1 .. (MYRANK+1)*maxnp

The restart point is after ``curnt`` of the last step and before its
``fields``; ``cont`` then calls ``fields`` once (pic/cont.f90:97) and the
main loop carries on.  :func:`save` / :func:`load` do the same for an
:class:`~maccpic_b200.em2.Em2Gpu` (or any object with get/set_fields and
get/set_particles), so runs can move between em2 and this library.

:func:`save_compact` / :func:`load_compact` keep the same state in one
``.npz`` of FP64 arrays (fields, each species in slot order, the step
counter and the grid size): half the bytes of em2's files, whose particle
files frame every 8-byte value with 8 bytes of record markers.
"""
from __future__ import annotations

import os

import numpy as np

FLD_ORDER = ["bx", "by", "bz", "ex", "ey", "ez"]                  # pic/output.f90:302-309
RHOJ_ORDER = ["rho", "jxm", "jxp", "jym", "jyp", "jzm", "jzp"]   # pic/output.f90:289-297
PART_FILES = ["x", "y", "vx", "vy", "vz", "g"]                   # pic/output.f90:312-364
FIELD_ID = {n: i for i, n in enumerate(
    ["ex", "ey", "ez", "bx", "by", "bz", "rho", "jxm", "jxp", "jym", "jyp", "jzm", "jzp"])}


def write_records(path: str, arrays) -> None:
    """One sequential record per array (4-byte length, data, 4-byte length)."""
    with open(path, "wb") as f:
        for a in arrays:
            b = np.ascontiguousarray(a, dtype="<f8").tobytes()
            if len(b) >= 2 ** 31:
                raise ValueError("record too large for a 4-byte length marker")
            n = np.array([len(b)], dtype="<i4").tobytes()
            f.write(n)
            f.write(b)
            f.write(n)


def read_records(path: str, count: int, length: int) -> list:
    """Read `count` records of `length` doubles, checking both markers."""
    out = []
    with open(path, "rb") as f:
        for k in range(count):
            head = np.frombuffer(f.read(4), dtype="<i4")
            if head.size != 1 or head[0] != 8 * length:
                raise ValueError(f"{path}: record {k} has length {head} bytes, "
                                 f"expected {8 * length}")
            data = np.frombuffer(f.read(8 * length), dtype="<f8").copy()
            tail = np.frombuffer(f.read(4), dtype="<i4")
            if tail.size != 1 or tail[0] != head[0]:
                raise ValueError(f"{path}: record {k} is truncated or corrupt")
            out.append(data)
    return out


_PER_PARTICLE = np.dtype([("h", "<i4"), ("v", "<f8"), ("t", "<i4")])


def write_particle_file(path: str, values_per_species) -> None:
    """One 8-byte record per particle (pic/output.f90:312-319)."""
    vals = np.concatenate([np.asarray(v, dtype=np.float64) for v in values_per_species])
    rec = np.empty(vals.size, dtype=_PER_PARTICLE)
    rec["h"] = 8
    rec["v"] = vals
    rec["t"] = 8
    rec.tofile(path)


def read_particle_file(path: str, counts) -> list:
    total = int(sum(counts))
    rec = np.fromfile(path, dtype=_PER_PARTICLE)
    if rec.size != total:
        raise ValueError(f"{path}: {rec.size} particle records, expected {total}")
    if not (np.all(rec["h"] == 8) and np.all(rec["t"] == 8)):
        raise ValueError(f"{path}: corrupt record markers")
    out, k = [], 0
    for c in counts:
        out.append(rec["v"][k:k + c].copy())
        k += c
    return out


def write_restart(directory: str, fields13: np.ndarray, parts, rank: int = 0) -> None:
    """fields13: (13, ny+3, nx+3) in FIELD_ID order; parts: list of (6, n)."""
    os.makedirs(directory, exist_ok=True)
    write_records(os.path.join(directory, "rhoj.fin"),
                  [fields13[FIELD_ID[n]] for n in RHOJ_ORDER])
    write_records(os.path.join(directory, "fld.fin"),
                  [fields13[FIELD_ID[n]] for n in FLD_ORDER])
    for k, name in enumerate(PART_FILES):
        write_particle_file(os.path.join(directory, f"{name}_rank{rank:03d}.fin"),
                            [p[k] for p in parts])


def read_restart(directory: str, nx: int, ny: int, counts, rank: int = 0):
    """-> (fields13, parts) with parts a list of (6, n) per species."""
    w = (nx + 3) * (ny + 3)
    fld = np.zeros((13, ny + 3, nx + 3))
    for name, a in zip(FLD_ORDER, read_records(os.path.join(directory, "fld.fin"), 6, w)):
        fld[FIELD_ID[name]] = a.reshape(ny + 3, nx + 3)
    for name, a in zip(RHOJ_ORDER, read_records(os.path.join(directory, "rhoj.fin"), 7, w)):
        fld[FIELD_ID[name]] = a.reshape(ny + 3, nx + 3)
    cols = [read_particle_file(os.path.join(directory, f"{name}_rank{rank:03d}.fin"), counts)
            for name in PART_FILES]
    parts = [np.stack([cols[k][s] for k in range(6)]) for s in range(len(counts))]
    for p in parts:
        if not np.all(np.isfinite(p)):
            raise ValueError("restart particles hold non-finite values")
    return fld, parts


def save(run, directory: str, rank: int = 0) -> None:
    """Write an Em2Gpu's state in em2's restart format (call after curnt)."""
    nsp = run.p.nsp
    write_restart(directory, run.get_fields(), [run.get_particles(s) for s in range(nsp)],
                  rank)


def load(run, directory: str, counts, rank: int = 0) -> None:
    """Read em2 restart files into an Em2Gpu; the caller then runs
    fields(it0+1) as ``cont`` does (pic/cont.f90:97)."""
    fld, parts = read_restart(directory, run.p.nx, run.p.ny, counts, rank)
    run.set_fields(fld)
    for s, p in enumerate(parts):
        run.set_particles(s, p)


def save_compact(run, path: str) -> None:
    """The run's whole state in one .npz: the 13 field arrays, every
    species' (x, y, vx, vy, vz, gamma) in slot order, the step counter and
    the grid.  `run` is an Em2Gpu or any object with get_fields,
    get_particles, p (nx, ny, nsp) and it."""
    nsp = run.p.nsp
    arrays = {"fields": run.get_fields(), "it": np.int64(run.it),
              "grid": np.array([run.p.nx, run.p.ny], dtype=np.int64)}
    for s in range(nsp):
        arrays[f"species{s}"] = run.get_particles(s)
    tmp = path + ".part.npz"
    np.savez(tmp, **arrays)
    os.replace(tmp, path)  # a reader never sees a half-written file


def load_compact(run, path: str) -> None:
    """Restore a state written by save_compact into `run`, which must have
    the same grid and species count; the step counter comes back too."""
    with np.load(path) as z:
        nx, ny = (int(v) for v in z["grid"])
        if (nx, ny) != (run.p.nx, run.p.ny):
            raise ValueError(f"checkpoint grid {nx}x{ny} differs from the run's "
                             f"{run.p.nx}x{run.p.ny}")
        nsp = sum(1 for k in z.files if k.startswith("species"))
        if nsp != run.p.nsp:
            raise ValueError(f"checkpoint holds {nsp} species, the run {run.p.nsp}")
        fld = z["fields"]
        if fld.shape != (13, ny + 3, nx + 3) or not np.all(np.isfinite(fld)):
            raise ValueError("checkpoint fields have the wrong shape or non-finite values")
        parts = [z[f"species{s}"] for s in range(nsp)]
        for p in parts:
            if p.ndim != 2 or p.shape[0] != 6 or not np.all(np.isfinite(p)):
                raise ValueError("checkpoint particles have the wrong shape or non-finite values")
        it = int(z["it"])
    run.set_fields(fld)
    for s, p in enumerate(parts):
        run.set_particles(s, p)
    run.it = it
