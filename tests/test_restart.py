"""em2's restart format (pic/output.f90:279-364, pic/cont.f90:21-92): record
framing, round trips, corrupt files, and a straight run against a run split
at a restart -- byte for byte on the oracle, as the reference's own restart
test demands of ccp1d (ccp1d/tests/restart/run.sh:1-29)."""
import numpy as np
import pytest


def test_record_framing(tmp_path):
    from maccpic_b200 import dumpio
    a = np.arange(10.0)
    p = tmp_path / "f.fin"
    dumpio.write_records(str(p), [a, 2 * a])
    raw = p.read_bytes()
    assert len(raw) == 2 * (4 + 80 + 4)
    assert np.frombuffer(raw[:4], "<i4")[0] == 80
    assert np.frombuffer(raw[84:88], "<i4")[0] == 80
    back = dumpio.read_records(str(p), 2, 10)
    np.testing.assert_array_equal(back[1], 2 * a)
    dumpio.write_particle_file(str(p), [np.array([1.5, 2.5]), np.array([3.5])])
    raw = p.read_bytes()
    assert len(raw) == 3 * 16
    assert np.frombuffer(raw[4:12], "<f8")[0] == 1.5


def test_corrupt_files_are_rejected(tmp_path):
    from maccpic_b200 import dumpio
    p = tmp_path / "f.fin"
    dumpio.write_records(str(p), [np.zeros(8)])
    raw = bytearray(p.read_bytes())
    with pytest.raises(ValueError):
        dumpio.read_records(str(p), 1, 9)          # wrong length
    p.write_bytes(bytes(raw[:-2]))
    with pytest.raises(ValueError):
        dumpio.read_records(str(p), 1, 8)          # truncated
    raw[-1] ^= 0xFF
    p.write_bytes(bytes(raw))
    with pytest.raises(ValueError):
        dumpio.read_records(str(p), 1, 8)          # bad trailing marker


def _case(oracle):
    from maccpic_b200 import loader
    cfg = loader.HarrisConfig(nx=32, ny=24, ppc=6, seed=9)
    fld, parts = loader.initial_state(cfg)
    rp = cfg.run_params()
    op = oracle.Params(nx=cfg.nx, ny=cfg.ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, qm=rp.qm, q=rp.q,
                       dn=rp.dn, am=rp.am, isav=4)
    return op, fld, parts


def test_split_run_through_restart_files_is_bitwise(tmp_path, oracle_lib):
    from maccpic_b200 import dumpio
    op, fld, parts = _case(oracle_lib)
    n1, n2 = 7, 6
    straight = oracle_lib.State(op, fld, parts)
    for it in range(1, n1 + n2 + 1):
        straight.move()
        straight.curnt()
        straight.fields(it)
    # first run: n1 steps, the last one stops after curnt and writes (output at it == nt)
    a = oracle_lib.State(op, fld, parts)
    for it in range(1, n1):
        a.move()
        a.curnt()
        a.fields(it)
    a.move()
    a.curnt()
    dumpio.write_restart(str(tmp_path), a.fld, a.parts)
    # second run: cont reads, then fields(it0+1) and the loop goes on
    counts = [p.shape[1] for p in parts]
    fld2, parts2 = dumpio.read_restart(str(tmp_path), op.nx, op.ny, counts)
    b = oracle_lib.State(op, fld2, parts2)
    b.fields(n1)
    for it in range(n1 + 1, n1 + n2 + 1):
        b.move()
        b.curnt()
        b.fields(it)
    np.testing.assert_array_equal(b.fld, straight.fld)
    for s in range(2):
        np.testing.assert_array_equal(b.parts[s], straight.parts[s])


class _HostRun:
    """A stand-in with the interface save_compact / load_compact use."""

    def __init__(self, nx, ny, nsp, fld=None, parts=None, it=0):
        class P:
            pass
        self.p = P()
        self.p.nx, self.p.ny, self.p.nsp = nx, ny, nsp
        self.fld = fld if fld is not None else np.zeros((13, ny + 3, nx + 3))
        self.parts = parts if parts is not None else [np.zeros((6, 0))] * nsp
        self.it = it

    def get_fields(self):
        return self.fld.copy()

    def set_fields(self, f):
        self.fld = np.array(f, copy=True)

    def get_particles(self, s):
        return self.parts[s].copy()

    def set_particles(self, s, p):
        self.parts = list(self.parts)
        self.parts[s] = np.array(p, copy=True)


def test_compact_checkpoint_round_trip(tmp_path):
    from maccpic_b200 import dumpio
    rng = np.random.default_rng(4)
    fld = rng.normal(size=(13, 11, 19))
    parts = [rng.normal(size=(6, 3000)), rng.normal(size=(6, 5))]
    a = _HostRun(16, 8, 2, fld, parts, it=123)
    path = str(tmp_path / "state.npz")
    dumpio.save_compact(a, path)
    b = _HostRun(16, 8, 2)
    dumpio.load_compact(b, path)
    np.testing.assert_array_equal(b.fld, fld)
    for x, y in zip(b.parts, parts):
        np.testing.assert_array_equal(x, y)
    assert b.it == 123
    # about half of em2's restart bytes once particles dominate (em2's
    # particle files frame every 8-byte value with 8 bytes of markers)
    dumpio.write_restart(str(tmp_path / "em2"), fld, parts)
    em2_bytes = sum(f.stat().st_size for f in (tmp_path / "em2").iterdir())
    assert (tmp_path / "state.npz").stat().st_size < 0.75 * em2_bytes


def test_compact_checkpoint_rejects_mismatches(tmp_path):
    from maccpic_b200 import dumpio
    a = _HostRun(16, 8, 2, parts=[np.ones((6, 3)), np.ones((6, 2))])
    path = str(tmp_path / "s.npz")
    dumpio.save_compact(a, path)
    with pytest.raises(ValueError):
        dumpio.load_compact(_HostRun(16, 9, 2), path)   # other grid
    with pytest.raises(ValueError):
        dumpio.load_compact(_HostRun(16, 8, 1), path)   # other species count
    bad = _HostRun(16, 8, 2, parts=[np.full((6, 3), np.nan), np.ones((6, 2))])
    dumpio.save_compact(bad, path)
    with pytest.raises(ValueError):
        dumpio.load_compact(_HostRun(16, 8, 2), path)   # non-finite particles
