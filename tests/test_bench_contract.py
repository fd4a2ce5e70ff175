"""The JSON line of ``bench.py --impl reference`` (the CPU reference arm), on
the CPU: one line with the contract's keys, printed by rank 0 alone when
launched as two ranks under torch.distributed.run."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "1", "--config",
        "harris_256x128_ppc16"]


def _json_lines(stdout):
    return [json.loads(l) for l in stdout.splitlines() if l.startswith("{")]


def _check_line(d, n_gpus):
    assert d["impl"] == "reference"
    assert d["metric"] == "particle-steps/s" and d["unit"] == "particle-steps/s"
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["n_gpus"] == n_gpus and d["steps"] == 1 and d["warmup"] == 1
    assert d["higher_is_better"] is True and d["scaling"] == "weak"
    assert d["config"]["workload"] == "harris_256x128_ppc16"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py", *ARGS], cwd=ROOT, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_line(lines[0], 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(300)
def test_reference_arm_under_two_ranks_prints_from_rank_zero_only():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--gpus", "2", *ARGS]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_line(lines[0], 2)


def test_roofline_inputs_are_consistent():
    """The push's committed DRAM traffic (profiles/, from an ncu capture) lies
    within 15 % of the algorithmic bytes the bench divides by the launch
    time (n x 48 B + W x 4 B x 20 at 2048x1024, 64 per cell): traffic far
    above them would mean re-reads, far below a capture of another kernel.
    The HBM peak is read from the measured figure when there is one."""
    import bench
    t = bench.profile_traffic("k_push_cells_f32_harris_2048x1024_ppc64")
    n = 2048 * 1024 * 64
    w = 2051 * 1027
    alg = n * 48 + w * 4 * 20
    assert t is not None and 0.85 < t / alg < 1.15
    peak, kind = bench.peaks()
    assert peak > 1000 and kind in ("measured", "fallback")
    assert bench.profile_traffic("no_such_kernel") is None
