#!/usr/bin/env python
"""Throughput of em2's time step on B200: particle-steps/s.

One step is em2's main-loop pass move -> curnt -> it+1 -> fields
(pic/main.f90:154-169) over the whole synthetic double-Harris workload
(default 2048x1024 cells, 64 particles per cell per species, 268M
particles), run through libem2g.  Prints one JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--config NAME] [--precision fp32|fp64]

value : device-resident state, K steps of em2g_step timed with CUDA events on
        the library's stream (inputs of 13-26 GB are far larger than L2), in
        the mixed-precision form by default; the FP64 form is then run from
        the same initial state for the same steps and reported beside it
        ("mixed_vs_fp64": its speed and the field-energy error between them).
e2e   : the same K steps through the drop-in entry points (em2g_move_curnt,
        em2g_fields) starting from the state in pinned host memory: the
        timed region includes the host->device upload of every field and
        particle array, a device->host read of ake / CG count / energies each
        step, and the download of the whole final state.
--impl reference : the CPU restatement of em2 (oracle/, pthreads on all host
        cores, one thread per em2 rank as em2's particle decomposition runs)
        on the same workload; bounded to at most 1 warm-up and 2 timed steps.
N > 1 : one process per GPU in em2's particle decomposition: each rank holds
        the whole grid and a full workload of particles (weak scaling), and
        rho/J and the kinetic energies are summed over ranks with an NCCL
        allreduce every step (pic/curnt.f90:363-376); time = max over ranks.
--only-adjoint, --only-ensemble : one leg alone, printed as its own JSON
        object (for profiling); --only-ensemble with --variant V and
        --sort-interval K skips the autotuner.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", default="harris_2048x1024_ppc64")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp32")
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--compare-steps", type=int, default=None,
                    help="length of the FP32-vs-FP64 comparison (default: the workload's "
                         "own step count)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--variant", type=int, default=None,
                    help="push variant to use instead of running the autotuner")
    ap.add_argument("--sort-interval", type=int, default=1,
                    help="sort interval to use with --variant")
    ap.add_argument("--only-adjoint", action="store_true",
                    help="run only the adjoint leg and print its JSON")
    ap.add_argument("--only-ensemble", action="store_true",
                    help="run only the ensemble leg and print its JSON (with --variant and "
                         "--sort-interval: those, without the autotuner)")
    # the 512x256 workload's adjoint: 800 steps, checkpoints every 50
    ap.add_argument("--stencils", type=int, choices=[0, 1], default=0,
                    help="Yee and smooth2 stages: 0 direct loads (the faster at every "
                         "measured size, the default), 1 TMA-staged tiles")
    ap.add_argument("--adjoint-steps", type=int, default=800)
    ap.add_argument("--adjoint-checkpoint", type=int, default=50)
    return ap.parse_args()


def dist_init():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """SM clocks and throttle reasons during a region: NVML read-only queries
    every 5 ms from a thread (the device found by its UUID, since NVML
    numbers GPUs without regard to CUDA_VISIBLE_DEVICES), or nvidia-smi
    sampling when NVML is missing."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.nvml = None
        self.sm, self.smax, self.reasons = [], None, set()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(
                uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _sample(self):
        nv, h = self.nvml
        try:
            self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            mask = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            for name, bit in self.REASONS:
                if mask & bit:
                    self.reasons.add(name)
        except Exception:
            pass

    def _loop(self):
        while not self.done.wait(0.005):
            self._sample()

    def __enter__(self):
        import threading
        try:
            self.nvml = self._nvml_handle()
        except Exception:
            self.nvml = None
        if self.nvml is not None:
            self.done = threading.Event()
            self._sample()
            self.thread = threading.Thread(target=self._loop, daemon=True)
            self.thread.start()
            return self
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.nvml is not None:
            self.done.set()
            self.thread.join()
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
            return
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            for ln in out.splitlines():
                f = [x.strip() for x in ln.split(",")]
                if len(f) < 9:
                    continue
                try:
                    self.sm.append(float(f[1]))
                    self.smax = float(f[2])
                except ValueError:
                    continue
                for (name, _), val in zip(self.REASONS, f[5:9]):
                    if val.lower() == "active":
                        self.reasons.add(name)

    def summary(self):
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.smax,
                "reasons": sorted(self.reasons), "samples": len(self.sm),
                "source": "nvml" if self.nvml is not None else "nvidia-smi"}


def peaks():
    """Measured HBM copy bandwidth (GB/s) from MEASURED_PEAKS.json: a number,
    or an object holding one (burst figure first: the push is timed per
    launch); 6650 GB/s, labelled "fallback", when there is none."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            v = json.load(f)["hbm_gbs"]
        if isinstance(v, dict):
            v = next(v[k] for k in ("burst", "value", "gbs", "sustained") if k in v)
        v = float(v)
        if v > 0:
            return v, "measured"
    except (OSError, ValueError, KeyError, TypeError, StopIteration):
        pass
    return 6650.0, "fallback"


def profile_traffic(kernel_key):
    """DRAM bytes per launch of the push kernel from the committed ncu summary
    (profiles/<kernel_key>.json), or None."""
    p = os.path.join(ROOT, "profiles", kernel_key + ".json")
    if not os.path.exists(p):
        return None
    try:
        return float(json.load(open(p))["dram_bytes_per_launch"])
    except (KeyError, ValueError):
        return None


def cpu_baseline(cfg, fields, parts_host):
    """The oracle (pthreads, all cores) on the whole workload, as the
    reference arm runs it: one untimed step, then one full step timed (the
    grid's serial field solve and every particle; about 15 s each on 16
    cores at 2048x1024)."""
    import oracle
    cores = os.cpu_count() or 1
    rp = cfg.run_params()
    op = oracle.Params(nx=rp.nx, ny=rp.ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, qm=rp.qm,
                       q=rp.q, dn=rp.dn, am=rp.am, isav=rp.isav)
    st = oracle.State(op, fields, parts_host)
    st.step(nthreads=cores)  # warm-up
    t = time.perf_counter()
    st.step(nthreads=cores)
    el = time.perf_counter() - t
    n = sum(p.shape[1] for p in parts_host)
    return {"value": n / el, "unit": METRIC, "cores": cores, "kind": "port",
            "sample": f"1 full step of the {cfg.nx}x{cfg.ny} grid with all {n} particles after "
                      f"1 untimed step (C restatement of em2, {cores} threads, field solve "
                      f"serial as in every em2 rank)"}


def run_reference(args):
    import numpy as np
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    from maccpic_b200 import loader
    cfg = loader.PRESETS[args.config]
    fields = loader.initial_fields(cfg)
    # the state is drawn on the GPU when there is one (set-up, not timed)
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    parts = [p.cpu().numpy() for p in loader.sample_particles_torch(cfg, device=dev)]
    rp = cfg.run_params()
    op = oracle.Params(nx=rp.nx, ny=rp.ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, qm=rp.qm,
                       q=rp.q, dn=rp.dn, am=rp.am, isav=rp.isav)
    st = oracle.State(op, fields, parts)
    del parts
    cores = os.cpu_count() or 1
    warm, steps = min(args.warmup, 1), max(1, min(args.steps, 2))
    for _ in range(warm):
        st.step(nthreads=cores)
    t = time.perf_counter()
    for _ in range(steps):
        st.step(nthreads=cores)
    el = time.perf_counter() - t
    n_total = sum(p.shape[1] for p in st.parts)
    value = n_total * steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": ws, "steps": steps, "warmup": warm, "ms_per_step": 1e3 * el / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded double-Harris sampling)",
        "config": {"workload": args.config, "grid": [cfg.nx, cfg.ny], "ppc": cfg.ppc,
                   "particles": n_total, "mass_ratio": cfg.mass_ratio},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "port",
                         "sample": f"{steps} full steps after {warm} warm-up (C restatement "
                                   f"of em2; em2 itself needs gfortran+MPI, absent)"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


class ParticleSource:
    """The seeded particles of a workload on one GPU: drawn once and kept on
    the device when both species' FP64 state (96 bytes per particle pair)
    takes at most an eighth of the device's memory, otherwise drawn again
    slice by slice for every upload (the 4096x2048, 100-per-cell workload:
    80 GB of FP64 state beside a run of 80 GB FP32 or 175 GB FP64)."""

    def __init__(self, cfg, local):
        import torch
        from maccpic_b200 import loader
        self.cfg, self.device = cfg, f"cuda:{local}"
        self.n = cfg.nx * cfg.ny * cfg.ppc
        total = torch.cuda.get_device_properties(local).total_memory
        self.parts = None
        if 96 * self.n <= total // 8:
            self.parts = loader.sample_particles_torch(cfg, device=self.device)
            torch.cuda.synchronize()

    def load(self, g):
        import torch
        from maccpic_b200 import loader
        if self.parts is not None:
            for s in range(2):
                g.set_particles_device(s, self.parts[s])
            return
        for s in range(2):
            g.set_particles_slices(s, self.n, (sl[s] for sl in loader.sample_particles_torch_slices(
                self.cfg, device=self.device)))
        torch.cuda.empty_cache()

    def host(self):
        """Both species in pinned host memory (whole mode only)."""
        return [p.cpu().pin_memory() for p in self.parts]

    def free(self):
        import torch
        self.parts = None
        torch.cuda.empty_cache()


def precision_compare(args, cfg, local, src, fields, stream, tuned):
    """The mixed FP32 path against the FP64 path from one initial state over
    the workload's own length (or --compare-steps), every `every` steps:
    the energy of each field component (Ex, Ey, Ez, By, Bz, and Bx - Bx(0),
    since the static Harris Bx dominates the total), the total field energy,
    the reconnected flux of both sheets and the kinetic energy, each as the
    relative difference |FP32 - FP64| / |FP64|.  An FP64 run from another seed
    gives, for context, the spread that particle sampling alone produces."""
    import dataclasses
    import numpy as np
    import torch
    from maccpic_b200 import _lib
    from maccpic_b200.em2 import Em2Gpu
    steps = args.compare_steps or cfg.check_steps or cfg.steps
    every = max(1, min(50, steps))
    nx, ny = cfg.nx, cfg.ny
    bx0 = fields[3, 1:ny + 1, 1:nx + 1]
    names = ["ex", "ey", "ez", "by", "bz", "bx_minus_bx0", "field_total", "flux_sheet1",
             "flux_sheet2", "kinetic"]

    def series(precision, source):
        torch.cuda.empty_cache()
        rp = cfg.run_params(device=local, precision=precision)
        g = Em2Gpu(rp)
        try:
            g.set_stream(stream)
            g.set_fields(fields)
            source.load(g)
            if precision == _lib.FP32:
                g.set_variant(tuned["variant"])
                g.set_sort_interval(tuned["sort_interval"])
            out, t = [], 0.0
            done = 0
            while done < steps:
                k = min(every, steps - done)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                r = g.step(k)
                torch.cuda.synchronize()
                t += time.perf_counter() - t0
                done += k
                d = g.diagnostics()
                bx = g.get_field("bx")[1:ny + 1, 1:nx + 1]
                e = d["energies"]
                out.append([e[0], e[1], e[2], e[4], e[5],
                            0.5 * float(np.mean((bx - bx0) ** 2)), float(e.sum()),
                            d["flux"][0], d["flux"][1], float(np.sum(r["ake"]))])
            return np.array(out), t
        finally:
            g.close()

    q32, t32 = series(_lib.FP32, src)
    q64, t64 = series(_lib.FP64, src)
    other = ParticleSource(dataclasses.replace(cfg, seed=cfg.seed + 1), local)
    q64b, _ = series(_lib.FP64, other)
    other.free()
    rel = np.abs(q32 - q64) / np.abs(q64)
    spread = np.abs(q64b - q64) / np.abs(q64)
    return {"steps": steps, "every": every, "quantities": names,
            "max_rel_error": dict(zip(names, rel.max(0).tolist())),
            "final_rel_error": dict(zip(names, rel[-1].tolist())),
            "fp64_seed_spread_max": dict(zip(names, spread.max(0).tolist())),
            "fp64_seed_spread_final": dict(zip(names, spread[-1].tolist())),
            "fp32_ms_per_step": 1e3 * t32 / steps, "fp64_ms_per_step": 1e3 * t64 / steps,
            "final_fp64": dict(zip(names, q64[-1].tolist()))}


def stencil_compare(g, stream, calls=20, rounds=3):
    """The field solve alone (em2g_fields: fold, Yee, smooth2 of rho,
    Poisson/CG) on the run's final state, with each stencil implementation
    (direct loads, TMA-staged tiles), CUDA events on the run's stream; best
    of `rounds` rounds of `calls` calls, each call with its own host
    synchronisation."""
    import torch
    it = g.it + 1
    best = {}
    for _ in range(rounds):
        for mode in (0, 1):
            g.set_stencils(mode)
            g.fields(it)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(calls):
                g.fields(it)
            b.record(stream)
            torch.cuda.synchronize()
            best[mode] = min(best.get(mode, float("inf")), a.elapsed_time(b) / calls)
    g.set_stencils(0)
    return {"direct_ms_per_fields_call": best[0], "tma_ms_per_fields_call": best[1],
            "calls": calls, "rounds": rounds}


def measure(args, cfg, precision, local, src, fields, stream, ws, stencils=False):
    """Device-resident run: warm-up, then K timed steps.  Returns timings,
    counters and the final fields and kinetic energies; with `stencils`,
    also the field solve timed with each stencil implementation."""
    import torch
    from maccpic_b200 import _lib
    from maccpic_b200.em2 import Em2Gpu
    rp = cfg.run_params(device=local, precision=precision)
    if ws > 1:
        # every rank adds a full workload of particles (weak scaling of em2's
        # particle decomposition): the macro charge and mass scale by 1/N so
        # that the plasma is the same one, sampled N times more finely
        rp.q = [q / ws for q in rp.q]
        rp.am = [a / ws for a in rp.am]
    torch.cuda.empty_cache()
    g = Em2Gpu(rp)
    g.set_stream(stream)
    g.set_stencils(args.stencils)
    g.set_fields(fields)
    src.load(g)
    torch.cuda.synchronize()
    # the project's autotuner picks the push variant and the sort interval on
    # this state (its steps are part of the warm-up), unless they are given
    from maccpic_b200 import autotune
    if args.variant is None:
        tuned = autotune.autotune(g, particles=src.n, use_cache=False, cache=None)
    else:
        k = min(args.sort_interval, g.max_sort_interval())
        g.set_variant(args.variant)
        g.set_sort_interval(k)
        tuned = {"variant": args.variant, "name": g.variant()[1], "times_ms": None,
                 "sort_interval": k, "interval_ms": None}
    # back to the initial state, so that every measured run starts from it
    g.set_fields(fields)
    src.load(g)
    g.it = 0
    if ws > 1:
        from maccpic_b200.distributed import GpuBackend, ParticleDecomposition
        pd = ParticleDecomposition(GpuBackend(g))
        it = [0]

        def one_step():
            it[0] += 1
            return pd.step(it[0])
    else:
        def one_step():
            return g.step(1)
    for _ in range(args.warmup):
        one_step()
    g.reset_counters()
    g.set_timing(True)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(ws)
    torch.cuda.synchronize()
    cg = []
    with Clocks(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            r = one_step()
            cg.append(r["cg_iters"])
        stop.record(stream)
        torch.cuda.synchronize()
    barrier(ws)
    ms = max_over_ranks(ws, start.elapsed_time(stop))
    cnt = g.counters()
    g.set_timing(False)
    out = {"ms": ms, "counters": cnt, "cg": cg, "clocks": clk.summary(), "ake": r["ake"],
           "tuned": tuned}
    if stencils:
        out["stencils"] = stencil_compare(g, stream)
    g.close()
    return out


def run_ours(args):
    import numpy as np
    import torch
    from maccpic_b200 import build, loader, _lib

    ws, rank, local = dist_init()
    build.build()
    cfg = loader.PRESETS[args.config]
    fp32 = args.precision == "fp32"
    stream = torch.cuda.current_stream()
    fields = loader.initial_fields(cfg)
    n = cfg.nx * cfg.ny * cfg.ppc
    n_total = 2 * n
    W = (cfg.nx + 3) * (cfg.ny + 3)
    import dataclasses
    rank_cfg = dataclasses.replace(cfg, seed=cfg.seed * 1000 + rank)
    src = ParticleSource(rank_cfg, local)

    main = measure(args, cfg, _lib.FP32 if fp32 else _lib.FP64, local, src, fields, stream, ws,
                   stencils=ws == 1)
    ms = main["ms"]
    value = n_total * ws * args.steps / (ms / 1e3)
    # the FP64 path on the same initial state: its speed, timed as the main
    # run is, and (one rank) the mixed path's error against it over the
    # workload's whole length
    compare = None
    if fp32 and not args.no_fp64_compare:
        try:
            ref = measure(args, cfg, _lib.FP64, local, src, fields, stream, ws)
            compare = {"fp64_value": n_total * ws * args.steps / (ref["ms"] / 1e3),
                       "fp64_ms_per_step": ref["ms"] / args.steps,
                       "speedup_fp32_over_fp64": ref["ms"] / ms}
            if ws == 1:
                compare.update(precision_compare(args, cfg, local, src, fields, stream,
                                                 main["tuned"]))
        except _lib.Em2gError as exc:  # e.g. the FP64 state does not fit beside the run
            compare = {"fp64_unavailable": str(exc)}
            torch.cuda.empty_cache()
    whole = src.parts is not None
    parts_host = None
    if rank == 0 and whole and (not args.no_e2e or not args.no_cpu_baseline):
        parts_host = src.host()
    src.free()

    cnt = main["counters"]
    # roofline of the dominant kernel (the fused push of one species):
    # algorithmic bytes per launch = n * (particle state read + written) +
    # the grid arrays it touches (6 scaled field arrays read, 7 deposit
    # arrays read-modify-written) = W * word * (6 + 14)
    word = 4 if fp32 else 8
    per_particle = 48 if fp32 else 96
    bytes_launch = n * per_particle + W * word * 20
    avg_ms = cnt["push_ms"] / max(cnt["push_launches_timed"], 1)
    achieved = bytes_launch / (avg_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    kernel = "k_push_cells_f32" if fp32 else "k_push_cells_f64"
    traffic = profile_traffic(f"{kernel}_{args.config}")

    e2e = None
    if rank == 0 and whole and not args.no_e2e:
        rp = cfg.run_params(precision=_lib.FP32 if fp32 else _lib.FP64,
                            sort_interval=main["tuned"]["sort_interval"])
        e2e = run_e2e(args, cfg, rp, fields, parts_host, main["tuned"]["variant"])
    ens = None
    if rank == 0 and ws == 1 and fp32 and not args.no_ensemble:
        ens = run_ensemble(args, local)
    adj = None
    if rank == 0 and ws == 1 and not args.no_adjoint:
        adj = run_adjoint(args, local)
    cpu = None
    if rank == 0 and ws == 1 and whole and not args.no_cpu_baseline:
        cpu = cpu_baseline(cfg, fields, [p.numpy() for p in parts_host])
        del parts_host
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if fp32 else "f64",
            "data": "synthetic (seeded double-Harris sampling, GPU Philox)",
            "config": {"workload": args.config, "grid": [cfg.nx, cfg.ny], "ppc": cfg.ppc,
                       "particles_per_gpu": n_total, "mass_ratio": cfg.mass_ratio,
                       "precision": ("mixed: FP32 push/deposit/Yee, FP64 reductions"
                                     if fp32 else "FP64 (em2's arithmetic)"),
                       "path": "em2g_step (fused push, cell-sorted)",
                       "stencils": "TMA-staged tiles" if args.stencils else "direct loads",
                       "l2": f"inputs larger than L2 (particle state "
                             f"{n_total * per_particle / 2 / 1e9:.1f} GB)",
                       "parallelism": (f"particle decomposition x{ws} (grid replicated, "
                                       f"NCCL allreduce of rho/J and ake each step)"
                                       if ws > 1 else "1 GPU"),
                       "cg_iters_mean": sum(main["cg"]) / len(main["cg"]),
                       "push_variant": main["tuned"]["name"],
                       "variant_times_ms": main["tuned"]["times_ms"],
                       "sort_interval": main["tuned"]["sort_interval"],
                       "interval_step_ms": main["tuned"]["interval_ms"]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": kernel,
                         "peak_kind": peak_kind, "bytes_per_launch": bytes_launch,
                         "avg_launch_ms": avg_ms},
            "gpu_launches": cnt["kernel_launches"],
            "clocks": main["clocks"],
            "stencils": main.get("stencils"),
            "mixed_vs_fp64": compare,
            "adjoint_over_forward": adj["gradient_over_forward"] if adj else None,
            "adjoint": adj,
            "ensemble": ens,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_adjoint(args, local):
    """d(reconnected flux after T steps)/d(psi0, guide field, sheet
    thickness) on the 512x256, 32-ppc double-Harris workload: the FP64 CUDA
    step with the exact Poisson solve, T forward steps timed alone, then the
    whole gradient (recording forward sweep, reverse sweep, the initial-state
    map) timed the same way."""
    import torch
    from maccpic_b200 import adjoint as A, loader
    cfg = loader.PRESETS["harris_512x256_ppc32"]
    T, K = args.adjoint_steps, args.adjoint_checkpoint
    theta = (cfg.psi0_over_b0di, cfg.guide_over_b0, cfg.l_over_di)
    dev = f"cuda:{local}"
    d = A.make_draws(cfg, device=dev)
    k = A.step_const(cfg)

    def timed(fn):
        torch.cuda.synchronize()
        t = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t, out

    # one workspace (context, per-step E and B slots, checkpoints) for every
    # gradient below, as a caller computing many gradients keeps it; by
    # default it holds as many steps' E and B as half the free memory takes
    t_setup, ws = timed(lambda: A.CudaAdjoint(k, *A.initial_state_torch(cfg, theta, d), T, K,
                                              cfg.isav))
    try:
        slots = ws.field_slots()
        ws.g.step(2)
        ws.load(*A.initial_state_torch(cfg, theta, d))
        t_fwd, _ = timed(lambda: ws.g.step(T))
        A.theta_gradient_cuda(cfg, theta, min(T, 4), checkpoint=K, draws=d, workspace=ws)
        t_grad, (F, g) = timed(lambda: A.theta_gradient_cuda(cfg, theta, T, checkpoint=K,
                                                             draws=d, workspace=ws))
        ws.load(*A.initial_state_torch(cfg, theta, d))
        t_rec, _ = timed(lambda: ws.forward(T))
        Bf = ws.final_B()
        t_rev, _ = timed(lambda: ws.backward([torch.zeros_like(b) for b in Bf],
                                             [torch.ones_like(b) * 1e-3 for b in Bf]))
        # the same gradient in the least memory: K slots, every step before
        # the last K recomputed from its checkpoint in the reverse sweep
        ws.set_field_slots(K)
        A.theta_gradient_cuda(cfg, theta, min(T, 4), checkpoint=K, draws=d, workspace=ws)
        t_grad_min, (F2, g2) = timed(lambda: A.theta_gradient_cuda(
            cfg, theta, T, checkpoint=K, draws=d, workspace=ws))
        ws.load(*A.initial_state_torch(cfg, theta, d))
        ws.forward(T)
        Bf = ws.final_B()
        t_rev_min, _ = timed(lambda: ws.backward([torch.zeros_like(b) for b in Bf],
                                                 [torch.ones_like(b) * 1e-3 for b in Bf]))
        ws.set_field_slots(slots)
        # the gradient against central differences of the same forward
        # (h = 1e-3, common random numbers) at growing horizons
        fd = {}
        for t in sorted({min(T, x) for x in (50, 100, 200, 400, T)}):
            fd[t] = A.fd_check_cuda(cfg, theta, t, h=1e-3, checkpoint=K, draws=d, workspace=ws)
        # at T, smaller steps: a difference over +-1e-3 is no longer linear
        # after hundreds of steps of a kinetic plasma, one over +-1e-6 is
        fd_h = {h: A.fd_check_cuda(cfg, theta, T, h=h, checkpoint=K, draws=d, workspace=ws)
                for h in (1e-4, 1e-5, 1e-6)}
    finally:
        ws.close()
    torch.cuda.empty_cache()
    n = 2 * cfg.nx * cfg.ny * cfg.ppc
    w = (cfg.nx + 3) * (cfg.ny + 3)
    ck_bytes = 8 * -(-T // K) * (13 * w + 6 * n)
    slot_bytes = 8 * 6 * cfg.nx * cfg.ny
    agree = [t for t, r in fd.items() if max(r["rel_error"]) <= 0.01]
    return {"workload": "harris_512x256_ppc32", "particles": n,
            "steps": T, "checkpoint": K, "flux": F, "dflux_dtheta": [float(x) for x in g],
            "field_slots": slots, "recomputed_steps": max(0, T - slots),
            "forward_ms_per_step": t_fwd * 1e3 / T,
            "recording_forward_ms_per_step": t_rec * 1e3 / T,
            "reverse_ms_per_step": t_rev * 1e3 / T,
            "gradient_ms": t_grad * 1e3,
            "gradient_over_forward": t_grad / t_fwd,
            "workspace_setup_ms": t_setup * 1e3,
            "workspace_bytes": ck_bytes + slots * slot_bytes,
            "least_memory": {"field_slots": K, "recomputed_steps": max(0, T - K),
                             "gradient_over_forward": t_grad_min / t_fwd,
                             "gradient_ms": t_grad_min * 1e3,
                             "reverse_ms_per_step": t_rev_min * 1e3 / T,
                             "workspace_bytes": ck_bytes + K * slot_bytes,
                             "dflux_dtheta": [float(x) for x in g2]},
            "memory": "checkpoints every K steps (fields + particles); E and B of the last "
                      "field_slots steps kept by the forward sweep, every step before them "
                      "recomputed a segment at a time from its checkpoint in the reverse sweep",
            "fd_h": 1e-3,
            "fd_rel_error": max(fd[T]["rel_error"]),
            "fd": {str(t): r for t, r in fd.items()},
            "fd_agree_1pct_max_steps": max(agree) if agree else 0,
            "fd_at_T_by_h": {f"{h:g}": {"fd": r["fd"], "rel_error": r["rel_error"]}
                             for h, r in fd_h.items()},
            "fd_rel_error_at_T_smallest_h": max(fd_h[1e-6]["rel_error"]),
            "forward": "em2g_step FP64, exact (spectral) Poisson solve"}


def run_ensemble(args, local):
    """The uneven batch of double-Harris runs (64 runs, grids log-uniform
    from 128x64 to 1024x512, 16-64 particles per cell, mass ratio 25/49/100)
    as one ensemble: one graph launch per step."""
    import torch
    from maccpic_b200.ensemble import harris_ensemble, load_harris
    from maccpic_b200.autotune import autotune_ensemble
    cfgs = harris_ensemble(64, seed=0)
    ens = load_harris(cfgs, device=f"cuda:{local}")
    try:
        if args.only_ensemble and args.variant is not None:
            ens.set_variant(args.variant)
            ens.set_sort_interval(args.sort_interval)
            tuned = {"variant": args.variant, "sort_interval": args.sort_interval,
                     "times_ms": None, "interval_ms": None}
        else:
            tuned = autotune_ensemble(ens)  # the project's autotuner, on this batch
        def timed_steps():
            # warm-up: at least two regrouping cycles, so that the graph of
            # every kind of step is captured before the timing
            ens.step(max(args.warmup, 2 * tuned["sort_interval"]))
            start = torch.cuda.Event(enable_timing=True)
            stop = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            start.record()
            out = ens.step(args.steps)
            stop.record()
            torch.cuda.synchronize()
            return start.elapsed_time(stop), out, ens.counters()["kernels_per_step"]

        # one graph launch per step of the stage-by-stage kernels, then of the
        # single persistent launch that runs every stage
        ms_staged, out, k_staged = timed_steps()
        ens.set_fused(True)
        ms_fused, out_f, k_fused = timed_steps()
        phases = ens.phase_ms()
        fused = ms_fused <= ms_staged
        ms = ms_fused if fused else ms_staged
        out = out_f if fused else out
        n = ens.particles
        return {"workload": "harris_ensemble_64runs", "runs": len(cfgs), "particles": n,
                "grids": [min(c.nx for c in cfgs), max(c.nx for c in cfgs)],
                "value": n * args.steps / (ms / 1e3), "unit": METRIC,
                "ms_per_step": ms / args.steps, "graph": True,
                "step": "one persistent launch" if fused else "one launch per stage",
                "kernels_per_step": k_fused if fused else k_staged,
                "fused_ms_per_step": ms_fused / args.steps,
                "staged_ms_per_step": ms_staged / args.steps,
                "staged_kernels_per_step": k_staged,
                "fused_phase_ms": [round(x, 4) for x in phases if x > 0],
                "cg_iters_max": int(out["cg_iters"].max()),
                "push_variant": tuned["variant"], "variant_step_ms": tuned["times_ms"],
                "sort_interval": tuned["sort_interval"],
                "interval_step_ms": tuned["interval_ms"]}
    finally:
        ens.close()
        torch.cuda.empty_cache()


def run_e2e(args, cfg, rp, fields, parts_host, variant=0):
    """The drop-in path from host memory, as em2's main loop drives it through
    the Fortran shim: the state uploaded once from pinned FP64 host arrays,
    then K steps of em2g_move_curnt (ake read back) and em2g_fields (CG count
    and energies read back), with every field array and every particle
    downloaded into the caller's pinned buffers whenever em2 would call
    `output` (it % isav == 0, pic/main.f90:158-159) and after the last step.
    K is the run's step count but at least one output interval (isav steps),
    so that the one upload and the final download are spread over no fewer
    steps than em2's own loop spreads each output over."""
    import torch
    from maccpic_b200.em2 import Em2Gpu

    fields_pin = torch.from_numpy(fields).pin_memory()
    fnp = fields_pin.numpy()
    pnp = [p.numpy() for p in parts_host]
    g = Em2Gpu(rp)
    g.set_variant(variant)
    out_f = torch.empty_like(fields_pin).pin_memory().numpy()
    out_p = [torch.empty_like(p).pin_memory().numpy() for p in parts_host]
    # warm-up (not timed): one full pass
    g.set_fields(fnp)
    for s in range(2):
        g.set_particles(s, pnp[s])
    g.move_curnt()
    g.fields(1)
    torch.cuda.synchronize()
    downloads = 0
    t = time.perf_counter()
    g.set_fields(fnp)
    for s in range(2):
        g.set_particles(s, pnp[s])
    g.it = 0
    K = max(args.steps, rp.isav)
    for it in range(1, K + 1):
        g.move_curnt()
        if it % rp.isav == 0 or it == K:
            g.get_fields(out=out_f)
            for s in range(2):
                g.get_particles(s, out=out_p[s])
            downloads += 1
        g.fields(it)
    el = time.perf_counter() - t
    g.close()
    n_total = sum(p.shape[1] for p in pnp)
    state = fnp.nbytes + sum(p.nbytes for p in pnp)
    small = 8 * (2 + 6) + 4
    return {"value": n_total * K / el, "unit": METRIC, "steps": K,
            "h2d_bytes_per_step": state / K,
            "d2h_bytes_per_step": (state * downloads + small * K) / K,
            "downloads": downloads, "isav": rp.isav, "n_gpus": 1,
            "path": "em2g_set_fields/em2g_set_particles (pinned host, FP64 em2 layout) once, K x "
                    "(em2g_move_curnt, em2g_fields), em2g_get_fields/em2g_get_particles every "
                    "isav steps and at the end"}


def main():
    args = parse()
    if args.only_adjoint:
        from maccpic_b200 import build
        build.build()
        print(json.dumps({"adjoint": run_adjoint(args, 0)}), flush=True)
        return
    if args.only_ensemble:
        from maccpic_b200 import build
        build.build()
        print(json.dumps({"ensemble": run_ensemble(args, 0)}), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
