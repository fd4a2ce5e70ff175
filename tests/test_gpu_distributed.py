"""em2's particle decomposition on the GPU data plane, one rank: the NCCL
allreduce of rho/J and ake (pic/curnt.f90:363-376, pic/move.f90:214) over
the __cuda_array_interface__ views GpuBackend takes of the library's field
block.  With one rank the sum is the identity, so the decomposed step must
give what a plain context gives, and the views must alias the library's
rho, jxm, jym and jzm arrays.  The rank runs in a child process (spawn) so
that its process group cannot outlive the test."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

STEPS = 6


def _case(precision):
    from maccpic_b200 import loader
    cfg = loader.HarrisConfig(nx=64, ny=48, ppc=8, seed=9)
    fld, parts = loader.initial_state(cfg)
    return cfg.run_params(precision=precision), fld, parts


def _worker(rank, port, precision, out):
    import datetime
    import torch
    import torch.distributed as dist
    from maccpic_b200 import build
    from maccpic_b200.distributed import GpuBackend, ParticleDecomposition
    from maccpic_b200.em2 import Em2Gpu
    build.build()
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                            world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        rp, fld, parts = _case(precision)
        g = Em2Gpu(rp)
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        be = GpuBackend(g)
        # the views alias the library's arrays: rho and jxm, jym, jzm
        g.move_curnt()
        torch.cuda.synchronize()
        w = (rp.nx + 3) * (rp.ny + 3)
        v = [t.double().cpu().numpy() for t in be.deposits()]
        alias = [np.array_equal(v[0][:w], g.get_field("rho").ravel()),
                 np.array_equal(v[0][w:], g.get_field("jxm").ravel()),
                 np.array_equal(v[1], g.get_field("jym").ravel()),
                 np.array_equal(v[2], g.get_field("jzm").ravel()),
                 not g.get_field("jxp").any()]
        g.close()
        g = Em2Gpu(rp)
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        pd = ParticleDecomposition(GpuBackend(g))
        akes = [pd.step(it)["ake"] for it in range(1, STEPS + 1)]
        torch.cuda.synchronize()
        np.savez(out, fld=g.get_fields(), ake=np.array(akes), alias=np.array(alias))
        g.close()
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_one_rank_nccl_decomposition_matches_plain_context(gpu, tmp_path, precision):
    from maccpic_b200.em2 import Em2Gpu
    out = str(tmp_path / "r.npz")
    mp.start_processes(_worker, args=(_free_port(), precision, out), nprocs=1, join=True,
                       start_method="spawn")
    got = np.load(out)
    assert got["alias"].all(), got["alias"]
    rp, fld, parts = _case(precision)
    with Em2Gpu(rp) as g:
        g.set_fields(fld)
        for s, p in enumerate(parts):
            g.set_particles(s, p)
        akes = []
        for it in range(1, STEPS + 1):
            akes.append(g.move_curnt())
            g.fields(it)
        ref = g.get_fields()
    # the deposits' atomics may add in another order: FP64 to 1e-12, FP32 to
    # FP32 rounding growth, relative to each array's largest value
    tol = 1e-12 if precision == 0 else 1e-5
    for k in range(6):
        scale = max(np.abs(ref[k]).max(), 1e-300)
        assert np.abs(got["fld"][k] - ref[k]).max() / scale < tol, k
    np.testing.assert_allclose(got["ake"], np.array(akes), rtol=tol)
