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
