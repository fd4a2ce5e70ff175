"""em2's particle decomposition, two ranks on CPU (gloo): the same
orchestration that drives the GPUs (maccpic_b200.distributed), here over the
oracle as the per-rank backend.  Splitting the particles over two ranks and
summing rho/J and ake must reproduce the single-rank run to the summation
noise floor -- the idiom of the reference's own multi-rank deposit test
(ccp1d/tests/deposit/test_deposit.f90:3-5, ccp1d/Makefile:70)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


class OracleBackend:
    def __init__(self, state):
        import torch
        self.st = state
        self._dep = torch.from_numpy(self.st.fld[6:13])  # shares memory

    def move_curnt(self):
        ake = self.st.move()
        self.st.curnt()
        return ake

    def deposits(self):
        # the oracle deposits jm and jp separately, as em2 does: all 7 arrays
        return [self._dep]

    def fields(self, it):
        return self.st.fields(it)


def _case():
    import oracle
    from maccpic_b200 import loader
    cfg = loader.HarrisConfig(nx=48, ny=32, ppc=8, seed=5)
    fld, parts = loader.initial_state(cfg)
    rp = cfg.run_params()
    op = oracle.Params(nx=cfg.nx, ny=cfg.ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, qm=rp.qm, q=rp.q,
                       dn=rp.dn, am=rp.am, isav=rp.isav)
    return op, fld, parts


def _worker(rank, world, port, steps, out):
    import torch.distributed as dist
    import oracle
    from maccpic_b200.distributed import ParticleDecomposition, rank_slice
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    op, fld, parts = _case()
    mine = [p[:, rank_slice(p.shape[1], rank, world)] for p in parts]
    pd = ParticleDecomposition(OracleBackend(oracle.State(op, fld, mine)))
    akes = []
    for it in range(1, steps + 1):
        r = pd.step(it)
        akes.append(r["ake"])
    if rank == 0:
        np.save(out + "_fld.npy", pd.b.st.fld)
        np.save(out + "_ake.npy", np.array(akes))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_decomposition_matches_one_rank(tmp_path, oracle_lib):
    steps = 12
    out = str(tmp_path / "r")
    mp.start_processes(_worker, args=(2, _free_port(), steps, out), nprocs=2, join=True,
                       start_method="spawn")
    op, fld, parts = _case()
    st = oracle_lib.State(op, fld, parts)
    akes = [st.step()["ake"] for _ in range(steps)]
    got = np.load(out + "_fld.npy")
    for k in range(6):
        err = np.abs(got[k] - st.fld[k]).max() / np.abs(st.fld[k]).max()
        assert err < 1e-11, (k, err)
    np.testing.assert_allclose(np.load(out + "_ake.npy"), np.array(akes), rtol=1e-12)


def test_rank_slices_cover_every_slot():
    from maccpic_b200.distributed import rank_slice
    for n in (0, 1, 7, 1000):
        for world in (1, 2, 3, 8):
            covered = np.concatenate([np.arange(n)[rank_slice(n, r, world)]
                                      for r in range(world)])
            np.testing.assert_array_equal(covered, np.arange(n))
