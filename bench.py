#!/usr/bin/env python
"""Throughput of the RK3 large step on B200: cell-updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload c3|moist-c2|dry|ensemble|adjoint]

Default workload (c3): the Weisman-Klemp supercell start on 640x768x80 cells
(39.3 M) of a vertically stretched column (dx = dy = 100 m, stretch_z 1 from
20 m at the ground to 500 m aloft under a 20.8 km lid, dt = 0.6 s,
nsound = 8, so 3 + 4 + 8 = 15 acoustic small steps per large step;
open-radiative laterals), Kessler warm rain (equation set 2), WENO5
moisture on the final stage with the positive-definite chain, the
1.5-order TKE closure, in the reference's flat (terrain_flag=.false.)
operator family for a stretched Cartesian column.  One "step" is one full
moist RK3 large step: closure and held tendencies, three RK stages (moist
stage terms, momentum advection, buoyancy, the psolver=3 acoustic stage,
getdiv/getdivx, theta and qv/qc/qr advection and update, boundaries, TKE
advection), the Kessler transition and solve3, through the library's C ABI.
--workload moist-c2 is the same physics on the uniform 256x256x80 grid
(dx = 1 km, dz = 250 m, dt = 5 s, nsound = 10); --workload dry the
64x64x40 dry warm bubble on the serial-periodic lane (nsound 6);
--workload ensemble the 64 uneven members; --workload adjoint the gradient
of the warm-rain transport model on the 96x96x48 supercell (t_adj/t_fwd).

Inputs are device resident; the step is captured once as a CUDA graph and
replayed; L2 is flushed (a 256 MiB write) before every timed step, outside
its event pair.  Under torchrun every rank runs its own replica (weak
scaling, no collective on the data path) and the job time is the max over
ranks.

Also measured: e2e (the same steps with the prognostic fields copied from
pinned host memory before and back after every step), the per-kernel device
time of each kernel (library launch profiler, CUDA events on the launching
stream) for the roofline of the dominant kernel, and the CPU oracle on the
host cores as the CPU baseline.

--impl reference times the reference algorithm's CPU implementation on the
host cores: the C restatement of the reference's CPU twins in oracle/ (the
reference itself is Python/CuPy and cannot run on the GPU box), composed in
the same large-step schedule, with all host threads, on a bounded sub-block
of the same workload and the same metric.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s per RK3 step (fwd, adjoint, ensemble) and % of HBM roofline"
UNIT = "cell-updates/s"
WORKLOAD = "dry periodic RK3 trajectory, warm bubble 64x64x40 (dx=dy=1 km, dz=500 m, dt=6 s, nsound=6)"

# Algorithmic bytes of one full RK3 large step per cell-update (4-byte
# words, each compulsory field once read and once written per grid pass):
# dry, nsound = 6: 3*(8+6) + 20*11 + 2 = 264 words = 1,056 B;
# moist: 149 + 20 * (small steps) words (16 closure/held, 3*(16+23)
# pre-acoustic and scalar passes, 20 per acoustic small step, 14 Kessler,
# 2 ppx): 449 words = 1,796 B at nsound 8 (dt 0.6 s, 15 small steps, the
# 640x768x80 column), 529 words = 2,116 B at nsound 10 (19 small steps,
# 256x256x80 and the ensemble).
STEP_BYTES_PER_CELL = 1056
MOIST_SMALL_STEPS = 4 + 5 + 10
MOIST_STEP_BYTES_PER_CELL = 4 * (149 + 20 * MOIST_SMALL_STEPS)

# Algorithmic words per cell of one launch of each kernel: every full field
# the launch must read or write once (stencil re-reads, halo words and
# horizontally uniform 1-D profiles are not counted; 3-D base-state arrays
# that the API passes as full fields are counted once).
KERNEL_WORDS_PER_CELL = {
    # in: u v w th3d pp3d th0 pi0 rho0 rf0; out: thv piadv ppterm rru rrv rrw divx
    "traj_prepare_kernel": 16,
    # in: u v w rru rrv rrw divx th3d c1 c2 rr0 rrf0 rth0; out: uten vten wten
    "traj_momentum_kernel": 16,
    # in: ppx ppi ua va wa mh rr0 rf0 mf c1 c2 piadv thv ppterm; out: ppd pp3d u3d v3d w3d rru rrv rrw qk pk1 pk2 mm
    "sound_prep_kernel": 26,
    # in+out: u v rru rrv; in: ppd thv uten vten
    "sound_uv_kernel": 12,
    # in: u v piadv ppterm ppten qk pk1 pk2 mm wten; in+out: w pp3d rrw; out: ppd
    "sound_column_kernel": 17,
    # one whole acoustic stage: in u v uten vten rru rrv thv piadv ppten ppterm
    # qk pk1 pk2 mm wten w pp3d rrw ppd (19); out u v rru rrv w pp3d ppd rrw (8);
    # plus the ppd exchange word of each small step (nloop = 2, 3, 6: 11/3 on
    # average over the three stage launches of a large step)
    "sound_stage_fused_kernel": 27 + 11 / 3,
    # in+out: rru rrv rrw; in: th3d th0; out: sadv
    "traj_theta_prep_kernel": 9,
    # in: rru rrv rrw sadv tha c1 c2 rr0; out: divx thten th3d
    "traj_theta_kernel": 11,
    # moist step: terrain/open acoustic stage
    # in: u v w pp3d qk pk1 pk2 mm ppten ppterm piadv rr0 rrf0 wten rru rrv rrw; out: w pp3d ppd rru rrv rrw
    "tos_column_kernel": 23,
    # in: ppd thv uten vten gxu gyv u v; out: u v
    "tos_pgrad_kernel": 10,
    # flat column: in ppd thv uten vten u v; out u v
    "tos_flat_pgrad_kernel": 8,
    # in: ppx ppi ua va wa ppterm piadv c1 c2 rf0 rr0 thv; out: ppd pp3d rru rrv rrw u v w qk pk1 pk2 mm
    "tos_prepare_kernel": 24,
    # in: scalar rru rrv rrw divx rr0 c1 c2; out: tendency
    "scalar_advection5_kernel": 9,
    # in: u v w rru rrv rrw divx rho0 rf0 rrf0 c2 gz; in+out: uten vten wten
    "mom5_adv_kernel": 18,
}

PROGNOSTIC = ("ua", "u3d", "va", "v3d", "wa", "w3d", "ppi", "pp3d", "ppx", "tha", "th3d")


def load_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:  # noqa: BLE001
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self) -> None:
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self) -> None:
        assert self.proc is not None and self.proc.stdout is not None
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_step_rate(steps_min: int, seconds_target: float, threads: int) -> dict:
    """Time the CPU oracle on the workload on the host cores."""
    from gm1_b200.initial_state import DRY_BUBBLE_64, dry_periodic_state
    from oracle import periodic as orc

    c = DRY_BUBBLE_64
    orc.set_threads(threads)
    a = dry_periodic_state(c)
    p = dict(ni=c.ni, nj=c.nj, nk=c.nk, steps=1, dt=c.dt, nsound=c.nsound, dx=c.dx, dy=c.dy, dz=c.dz)
    orc.traj_steps(a, **p)  # warm-up
    n = 0
    t0 = time.perf_counter()
    while n < steps_min or time.perf_counter() - t0 < seconds_target:
        orc.traj_steps(a, **p)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": c.cells * n / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} RK3 large steps of the full 64x64x40 domain in {dt:.2f} s "
                      f"(C restatement of the reference NumPy twins, bit-identical to them)"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from gm1_b200.initial_state import DRY_BUBBLE_64, dry_periodic_state
    from oracle import periodic as orc

    c = DRY_BUBBLE_64
    orc.set_threads(threads)
    a = dry_periodic_state(c)
    p = dict(ni=c.ni, nj=c.nj, nk=c.nk, steps=1, dt=c.dt, nsound=c.nsound, dx=c.dx, dy=c.dy, dz=c.dz)
    for _ in range(args.warmup):
        orc.traj_steps(a, **p)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.traj_steps(a, **p)
    dt = time.perf_counter() - t0
    value = c.cells * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded dry warm bubble)",
        "config": {"workload": WORKLOAD, "cells": c.cells, "device": "host CPU"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} timed RK3 large steps of the full domain after {args.warmup} "
                                   "warm-up steps (C restatement of the reference NumPy twins)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# The moist workloads.  "c3": the Weisman-Klemp supercell on the 640x768x80
# stretched column (dx = dy = 100 m, stretch_z 1 from 20 m at the ground to
# 500 m aloft under a 20.8 km lid, reference dz 100 m, dt 0.6 s, nsound 8:
# 3 + 4 + 8 = 15 acoustic small steps, 149 + 20*15 = 449 words = 1,796 B per
# cell-update), the largest single-GPU configuration and the default.
# "moist-c2": the same physics on the uniform 256x256x80 grid (dx = 1 km,
# dz = 250 m, dt 5 s, nsound 10: 19 small steps, 529 words = 2,116 B).
STRETCH_C3 = dict(ztop_m=20800.0, str_bot_m=200.0, str_top_m=15800.0, dz_bot_m=20.0, dz_top_m=500.0)
MOIST_WORKLOADS = {
    "c3": {
        "grid": dict(ni=640, nj=768, nk=80, dx=100.0, dy=100.0, dz=100.0, dt=0.6, nsound=8),
        "column": STRETCH_C3,
        "small_steps": 3 + 4 + 8,
        "name": ("moist Weisman-Klemp supercell 640x768x80 on a stretched column (dx=dy=100 m, stretch_z=1 dz "
                 "20-500 m, lid 20.8 km, dt=0.6 s, nsound=8, Kessler eqtset 2, WENO5 moisture, TKE sgsmodel 1, "
                 "open-radiative laterals, flat terrain_flag=.false. operator family)"),
        "cpu_subblock": (64, 64, 80),
    },
    "moist-c2": {
        "grid": dict(ni=256, nj=256, nk=80, dx=1000.0, dy=1000.0, dz=250.0, dt=5.0, nsound=10),
        "column": None,
        "small_steps": 4 + 5 + 10,
        "name": ("moist Weisman-Klemp supercell 256x256x80 (dx=dy=1 km, dz=250 m, dt=5 s, nsound=10, Kessler "
                 "eqtset 2, WENO5 moisture, TKE sgsmodel 1, open-radiative laterals)"),
        "cpu_subblock": (64, 64, 80),
    },
}
MOIST_INIT = dict(seed=2, bubble_k=3.0, noise_k=0.1, bubble_radius_m=(10000.0, 1500.0), bubble_center_z_m=1500.0)
# step-start state a user passes in and reads back: the A-level prognostic
# fields (each copied into its RK-stage twin on the device) and ppx
MOIST_PROGNOSTIC = ("ua", "va", "wa", "ppi", "tha", "qa", "tkea", "ppx")
MOIST_STAGE_TWIN = {"ua": "u3d", "va": "v3d", "wa": "w3d", "ppi": "pp3d", "tha": "th3d", "qa": "q3d", "tkea": "tke3d"}


def moist_step_bytes(workload: str) -> int:
    """Algorithmic bytes of one moist RK3 large step per cell-update:
    (149 + 20 * small steps) words."""
    return 4 * (149 + 20 * MOIST_WORKLOADS[workload]["small_steps"])


def moist_state(workload: str, ni=None, nj=None, nk=None):
    """The GPU arm's starting state (the package's builder)."""
    from gm1_b200.moist_step import MoistStepConfig, StretchedColumnSpec, weisman_klemp_initial_state

    w = MOIST_WORKLOADS[workload]
    g = dict(w["grid"])
    g.update({k: v for k, v in (("ni", ni), ("nj", nj), ("nk", nk)) if v is not None})
    column = None if w["column"] is None else StretchedColumnSpec(**w["column"])
    cfg = MoistStepConfig(**g, column=column)
    host, metrics = weisman_klemp_initial_state(cfg, **MOIST_INIT)
    return cfg, host, metrics


def moist_state_cpu(workload: str, ni, nj, nk):
    """The CPU arms' starting state, built by the oracle's own initial-state
    restatement (the same words as moist_state; no CUDA library is loaded on
    the CPU baseline or the reference arm)."""
    from types import SimpleNamespace

    from oracle.moist_initial import weisman_klemp_initial_state

    w = MOIST_WORKLOADS[workload]
    column = None if w["column"] is None else SimpleNamespace(**w["column"])
    cfg = SimpleNamespace(**dict(w["grid"], ni=ni, nj=nj, nk=nk, alph=0.60, kdiv=0.10,
                                 lateral_sides=(2, 2, 2, 2), column=column))
    cfg.obc = 2 | (2 << 4) | (2 << 8) | (2 << 12)
    host, metrics = weisman_klemp_initial_state(cfg, **MOIST_INIT)
    return cfg, host, metrics


def moist_cpu_rate(workload: str, steps_min: int, seconds_target: float, threads: int,
                   warmup: int = 1) -> tuple[float, int, float]:
    """The oracle composition on a sub-block of the moist workload on the
    host cores: (cell-updates/s, steps, seconds)."""
    from oracle import periodic as orc
    from oracle.moist_composition import OracleMoistStep

    orc.set_threads(threads)
    cfg, host, metrics = moist_state_cpu(workload, *MOIST_WORKLOADS[workload]["cpu_subblock"])
    o = OracleMoistStep(cfg, host, metrics)
    for _ in range(warmup):
        o.step()
    n = 0
    t0 = time.perf_counter()
    while n < steps_min or time.perf_counter() - t0 < seconds_target:
        o.step()
        n += 1
    dt = time.perf_counter() - t0
    return cfg.ni * cfg.nj * cfg.nk * n / dt, n, dt


def run_reference_moist(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    # the ensemble's members run the 1 km physics of configuration 2: its
    # reference arm is that per-cell rate
    workload = args.workload if args.workload in MOIST_WORKLOADS else "moist-c2"
    w = MOIST_WORKLOADS[workload]
    value, n, dt = moist_cpu_rate(workload, args.steps, 0.0, threads, warmup=args.warmup)
    ni, nj, nk = w["cpu_subblock"]
    g = w["grid"]
    sample = (f"{n} moist RK3 large steps of a {ni}x{nj}x{nk} sub-block of the workload (same column, spacing, "
              f"dt, nsound and initial state) in {dt:.2f} s after {args.warmup} warm-up steps, on all {threads} "
              "host threads: the oracle's C restatements of the reference's CPU twins (and, where the reference "
              "has only CUDA text, of that text) composed in the large-step schedule")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / n,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Weisman-Klemp supercell start)",
        "config": {"workload": w["name"], "cells": g["ni"] * g["nj"] * g["nk"], "device": "host CPU",
                   "sample": f"{ni}x{nj}x{nk} sub-block per step"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _dist_setup():
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)

    def barrier():
        torch.cuda.synchronize(device)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(device)

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return rank, world, local, device, barrier, max_over_ranks


def run_moist(args) -> None:
    import torch
    import torch.distributed as dist

    from gm1_b200 import _native
    from gm1_b200.moist_step import NativeMoistLargeStep, upload

    rank, world, local, device, barrier, max_over_ranks = _dist_setup()
    wl = MOIST_WORKLOADS[args.workload]
    step_bytes = moist_step_bytes(args.workload)
    cfg, host, metrics = moist_state(args.workload)
    cells = cfg.ni * cfg.nj * cfg.nk
    stream = torch.cuda.Stream(device)
    dev_state, dev_metrics = upload(host, device), upload(metrics, device)
    # the step through the library's whole-step C entry point
    # (gm1b_moist_large_step): one call per step, captured once as a graph
    with torch.cuda.stream(stream):
        model = NativeMoistLargeStep(cfg, dev_state, dev_metrics, stream=stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            model.step()
        stream.synchronize()
        graph = torch.cuda.CUDAGraph()
        try:
            with torch.cuda.graph(graph, stream=stream):
                model.step()
            use_graph = True
        except Exception as exc:  # noqa: BLE001 - capture refused: time direct launches
            print(f"CUDA graph capture failed ({exc}); timing direct launches", file=sys.stderr)
            torch.cuda.synchronize(device)
            use_graph = False

        def step() -> None:
            if use_graph:
                graph.replay()
            else:
                model.step()

        for _ in range(args.warmup):
            step()
        stream.synchronize()

    # ---- timed region: K graph replays, L2 flushed before each ----------
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    with torch.cuda.stream(stream):
        for q in range(args.steps):
            flush.zero_()
            starts[q].record(stream)
            step()
            ends[q].record(stream)
    barrier()
    clocks = sampler.stop()
    total_ms = max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(starts, ends)))
    ms_per_step = total_ms / args.steps
    value = world * cells * args.steps / (total_ms * 1e-3)

    # ---- the same step with the closure's held tendencies on (SGS stress,
    # scalar diffusion and upper Rayleigh damping once per step): a second
    # handle on the same state, captured and timed the same way (stretched
    # columns only) --------------------------------------------------------
    stress_step = None
    if cfg.stretched:
        import dataclasses

        scfg = dataclasses.replace(cfg, sgs_diffusion=True, rayleigh=True, dissipative_heating=True)
        with torch.cuda.stream(stream):
            smodel = NativeMoistLargeStep(scfg, dev_state, dev_metrics, stream=stream)
            smodel.step()
            stream.synchronize()
            sgraph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(sgraph, stream=stream):
                smodel.step()
            for _ in range(2):
                sgraph.replay()
        s_start = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        s_end = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        barrier()
        with torch.cuda.stream(stream):
            for q in range(args.steps):
                flush.zero_()
                s_start[q].record(stream)
                sgraph.replay()
                s_end[q].record(stream)
        barrier()
        s_ms = max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(s_start, s_end))) / args.steps
        smodel.check()
        del sgraph
        smodel.close()
        stress_step = {"ms_per_step": s_ms, "value": world * cells / (s_ms * 1e-3), "unit": UNIT,
                       "note": "the same step with the closure's held tendencies on (MoistStepConfig.sgs_diffusion "
                               ", .rayleigh and .dissipative_heating: strain, gettau, turbu/turbv/turbw and turbs of "
                               "theta and qv/qc/qr once per step, the upper Rayleigh damping above 15 km, the "
                               "dissipative heating; added in every RK stage)"}

    # ---- per-kernel device time (eager steps, launch profiler on) -------
    # run operation by operation on one stream: the profiler's event pairs
    # time each launch alone only when launches do not overlap
    nprof = min(args.steps, 5)
    sequential = NativeMoistLargeStep(cfg, dev_state, dev_metrics, stream=stream, concurrent=False)
    _native.profiler_enable(True)
    with torch.cuda.stream(stream):
        for _ in range(nprof):
            flush.zero_()
            sequential.step()
    stream.synchronize()
    _native.profiler_enable(False)
    sequential.close()
    stats = _native.profiler_collect()
    launches_per_step = sum(s["launches"] for s in stats) / nprof
    top = stats[0]
    avg_ms = top["total_ms"] / top["launches"]
    peak, peak_kind = load_peaks()
    words = KERNEL_WORDS_PER_CELL.get(top["name"])
    achieved = None if words is None else words * 4 * cells / (avg_ms * 1e-3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "traffic_per_launch.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get(args.workload, {}).get(top["name"])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": None if achieved is None else achieved / peak, "traffic": traffic, "kernel": top["name"],
                "avg_launch_ms": avg_ms, "alg_bytes_per_launch": None if words is None else words * 4 * cells,
                "peak_source": f"{peak_kind} hbm_gbs"}
    tot = sum(x["total_ms"] for x in stats)
    kernel_share = {s["name"]: round(s["total_ms"] / tot, 4) for s in stats[:16]}

    # ---- e2e: prognostic fields in from pinned host memory, the step
    # through the C ABI, the fields out again, all inside the event pair ----
    pinned = {n: torch.from_numpy(host[n]).pin_memory() for n in MOIST_PROGNOSTIC}
    with torch.cuda.stream(stream):
        for n, t in pinned.items():
            t.copy_(dev_state[n], non_blocking=True)
    stream.synchronize()
    h2d = sum(t.numel() * 4 for t in pinned.values())
    e_start = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_end = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    with torch.cuda.stream(stream):
        for q in range(args.steps):
            flush.zero_()
            e_start[q].record(stream)
            for n, t in pinned.items():
                dev_state[n].copy_(t, non_blocking=True)
            for n, twin in MOIST_STAGE_TWIN.items():
                dev_state[twin].copy_(dev_state[n])
            model.step()  # the C-ABI call itself (gm1b_moist_large_step), not a graph replay
            for n, t in pinned.items():
                t.copy_(dev_state[n], non_blocking=True)
            e_end[q].record(stream)
    barrier()
    e2e_ms = max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(e_start, e_end)))
    e2e_value = world * cells * args.steps / (e2e_ms * 1e-3)

    status = model.check()  # raises on a failure word of any step taken
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, n, dt = moist_cpu_rate(args.workload, 3, 10.0, threads)
        ni, nj, nk = wl["cpu_subblock"]
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{n} moist RK3 large steps of a {ni}x{nj}x{nk} sub-block of the workload in {dt:.2f} s "
                         "(the oracle's C restatements of the reference CPU twins composed in the same schedule)"}
    del graph
    model.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Weisman-Klemp supercell start: isnd 5 column, iwnd 2 hodograph, +3 K bubble, "
                "U(+-0.1 K) noise from numpy default_rng(2))",
        "config": {"workload": wl["name"], "mode": "fwd", "cells": cells, "large_steps_per_timed_step": 1,
                   "acoustic_small_steps_per_step": wl["small_steps"],
                   "l2": "flushed before every timed step (256 MiB write, outside the event pair)",
                   "cuda_graph": use_graph, "lateral_boundaries": "open-radiative (wbc=ebc=sbc=nbc=2)",
                   "entry_point": "gm1b_moist_large_step (one C-ABI call per step, captured as a CUDA graph)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single domain"},
        "step_roofline": {"bytes_per_cell_update": step_bytes,
                          "achieved_gbs": step_bytes * value / world / 1e9,
                          "frac": step_bytes * value / world / 1e9 / peak},
        "status": {"max_courant": status["max_courant"], "satadj_nonconverged_cells": status["satadj_nonconverged_cells"],
                   "max_fall_substeps": status["max_fall_substeps"]},
        "roofline": roofline, "kernel_share": kernel_share,
        "gpu_launches": int(round(launches_per_step * args.steps)),
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
        "clocks": clocks,
    }
    if stress_step is not None:
        line["with_held_closure"] = stress_step
    print(json.dumps(line), flush=True)


def _kernel_roofline(stats, cells_per_launch_unit: float, peak: float, peak_kind: str) -> dict:
    """roofline of the kernel with the most device time: its algorithmic
    words per cell x cells per launch over its average launch time."""
    top = stats[0]
    avg_ms = top["total_ms"] / top["launches"]
    words = KERNEL_WORDS_PER_CELL.get(top["name"])
    alg = None if words is None else words * 4 * cells_per_launch_unit
    achieved = None if alg is None else alg / (avg_ms * 1e-3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "traffic_per_launch.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get("ensemble", {}).get(top["name"])
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": None if achieved is None else achieved / peak, "traffic": traffic, "kernel": top["name"],
            "avg_launch_ms": avg_ms, "alg_bytes_per_launch": alg, "peak_source": f"{peak_kind} hbm_gbs"}


def run_ensemble(args) -> None:
    """Configuration 5: uneven Weisman-Klemp members, batched (one CUDA graph
    per ensemble step over 8 streams) against the same members launched one
    by one; members sharded over ranks by cell count."""
    import torch
    import torch.distributed as dist

    from gm1_b200 import _native
    from gm1_b200.ensemble import ENSEMBLE_GRID, MoistEnsemble, ensemble_members, member_initial_state
    from gm1_b200.replicas import member_shard

    rank, world, local, device, barrier, max_over_ranks = _dist_setup()
    members = ensemble_members(args.members)
    cells_all = [m.cells for m in members]
    mine = [members[q] for q in member_shard(cells_all, rank, world)]
    my_cells = sum(m.cells for m in mine)
    total_cells = sum(cells_all)
    hosts = [member_initial_state(m) for m in mine]
    # the batched method picks each member grid shape's advection z-chunk
    # with the project's autotuner (once per shape); the plain method keeps
    # the kernels' defaults
    from gm1_b200.autotune import Autotuner

    tuner = Autotuner()
    t_tune = time.perf_counter()
    batched = MoistEnsemble(mine, device, streams=8, hosts=hosts, tuner=tuner)
    t_tune = time.perf_counter() - t_tune
    plain = MoistEnsemble(mine, device, streams=1, hosts=hosts)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    for _ in range(args.warmup):
        batched.step_eager()
        plain.step_eager()
    torch.cuda.synchronize(device)
    batched.capture()
    for _ in range(args.warmup):
        batched.replay()
    torch.cuda.synchronize(device)

    def timed(ens, fn, sampler=None):
        st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = 0.0
        barrier()
        if sampler is not None:
            sampler.start()
        for _ in range(args.steps):
            with torch.cuda.stream(ens.main):
                flush.zero_()
                st.record(ens.main)
            fn()
            with torch.cuda.stream(ens.main):
                en.record(ens.main)
            en.synchronize()
            ms += st.elapsed_time(en)
        barrier()
        clocks = sampler.stop() if sampler is not None else None
        return max_over_ranks(ms), clocks

    sampler = ClockSampler(local)
    b_ms, clocks = timed(batched, batched.replay, sampler)
    p_ms, _ = timed(plain, plain.step_eager)
    value = total_cells * args.steps / (b_ms * 1e-3)
    plain_value = total_cells * args.steps / (p_ms * 1e-3)

    # per-kernel device time of one plain step (launch profiler; the plain
    # ensemble launches one kernel at a time, so each event pair times one)
    _native.profiler_enable(True)
    plain.step_eager()
    torch.cuda.synchronize(device)
    _native.profiler_enable(False)
    stats = _native.profiler_collect()
    launches_per_step = sum(x["launches"] for x in stats)
    peak, peak_kind = load_peaks()
    # every member launches the top kernel equally often, so its average
    # launch covers the members' mean cell count
    roofline = _kernel_roofline(stats, my_cells / len(mine), peak, peak_kind)
    tot = sum(x["total_ms"] for x in stats)
    kernel_share = {x["name"]: round(x["total_ms"] / tot, 4) for x in stats[:12]}

    # e2e: each member's step-start state in from pinned host memory, out after
    pinned = [{n: torch.from_numpy(h[0][n]).pin_memory() for n in MOIST_PROGNOSTIC} for h in hosts]
    for ens_state, pin in zip(batched.steps, pinned):
        for n, t in pin.items():
            t.copy_(ens_state.s[n])
    h2d = sum(t.numel() * 4 for pin in pinned for t in pin.values())

    def e2e_step():
        with torch.cuda.stream(batched.main):
            for ens_state, pin in zip(batched.steps, pinned):
                for n, t in pin.items():
                    ens_state.s[n].copy_(t, non_blocking=True)
                for n, twin in MOIST_STAGE_TWIN.items():
                    ens_state.s[twin].copy_(ens_state.s[n])
        batched.replay()
        with torch.cuda.stream(batched.main):
            for ens_state, pin in zip(batched.steps, pinned):
                for n, t in pin.items():
                    t.copy_(ens_state.s[n], non_blocking=True)

    e_ms, _ = timed(batched, e2e_step)
    e2e_value = total_cells * args.steps / (e_ms * 1e-3)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, n, dt = moist_cpu_rate("moist-c2", 3, 10.0, threads)
        ni, nj, nk = MOIST_WORKLOADS["moist-c2"]["cpu_subblock"]
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{n} moist RK3 large steps of one {ni}x{nj}x{nk} domain in {dt:.2f} s (per-cell rate of "
                         "the oracle composition; every member runs the same per-cell work)"}
    batched.release()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    g = ENSEMBLE_GRID
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": b_ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic ({args.members} seeded Weisman-Klemp members, numpy default_rng(5))",
        "config": {"workload": f"ensemble of {args.members} uneven moist members (nx, ny in 48..160, nz in 40..64, "
                               f"dx=dy={g['dx'] / 1000:g} km, dz={g['dz']:g} m, dt={g['dt']:g} s, nsound={g['nsound']}, "
                               "bubble U[1,3] K jittered +-5 km, Kessler, WENO5, TKE, open-radiative laterals)",
                   "mode": "ensemble", "cells": total_cells, "members": args.members,
                   "batched": "one CUDA graph per ensemble step, members over 8 streams",
                   "autotune": {"shapes": len(tuner.table) // 2, "set_up_s": round(t_tune, 2),
                                "chunks": {k: v["best"] for k, v in list(tuner.table.items())[:8]}},
                   "plain_cell_updates_per_s": plain_value, "plain_ms_per_step": p_ms / args.steps,
                   "batched_over_plain": value / plain_value,
                   "l2": "flushed before every timed step (256 MiB write, outside the event pair)",
                   "parallelism": f"members sharded over {world} ranks by cell count" if world > 1 else "one GPU"},
        "step_roofline": {"bytes_per_cell_update": MOIST_STEP_BYTES_PER_CELL,
                          "achieved_gbs": MOIST_STEP_BYTES_PER_CELL * value / world / 1e9,
                          "frac": MOIST_STEP_BYTES_PER_CELL * value / world / 1e9 / peak},
        "roofline": roofline, "kernel_share": kernel_share,
        "gpu_launches": int(launches_per_step * args.steps),
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


# Configuration 4: the adjoint.  The warm-rain transport model of
# gm1_b200.adjoint (theta', qv, qc, qr under RK3 WENO5 transport by frozen
# mass fluxes, then collection and the single-pass saturation adjustment),
# linearised about a Weisman-Klemp supercell (warm bubble with cloud and
# rain water in its core) spun up for ADJOINT_SPINUP large steps of the full
# moist model on the 96x96x48 grid; J = the domain's condensate
# sum(rho0 (qc + qr)) at the end of the window.
ADJOINT_GRID = dict(ni=96, nj=96, nk=48, dx=1000.0, dy=1000.0, dz=300.0, dt=5.0, nsound=6)
ADJOINT_SPINUP = 60
ADJOINT_INIT = dict(seed=4, bubble_k=3.0, noise_k=0.1, bubble_radius_m=(10000.0, 1500.0), bubble_center_z_m=1500.0,
                    bubble_cloud=1.0e-3, bubble_rain=5.0e-4)
# forward words per cell-update: per scalar and RK stage the transport reads
# s_prev, s_0, rru, rrv, rrw, divx, rr0, c1, c2 and writes s_new (10 words,
# 4 scalars x 3 stages), the Kessler pieces read theta', qv, qc, qr, th0,
# pi0, pp3d, prs and write theta', qv, qc, qr (12): 132 words.  The adjoint
# step is 3 x that (one forward recompute from the checkpoint, the reverse
# reading the primal and the adjoint and writing the adjoint).
ADJOINT_FWD_WORDS = 4 * 3 * 10 + 12
ADJOINT_WORDS = 3 * ADJOINT_FWD_WORDS
KERNEL_WORDS_PER_CELL.update({
    # the advection adjoint's two passes; the 18 face-coefficient words per
    # cell that pass 1 writes and pass 2 reads are scratch, not counted
    # in: carrier rru rrv rrw c1 c2 rr0 tendency-adjoint
    "advection_adjoint_faces_kernel": 8,
    # in: tendency-adjoint rr0 divx accumulate; out: scalar-adjoint
    "advection_adjoint_gather_compact_kernel": 5,
    # in: scalar; out: carrier
    "scalar_carrier_open_kernel": 2,
    # in: th0 pi0 pp3d prs th3d qv qc g_th g_qv g_qc; out: g_th g_qv g_qc
    "satadj1_adjoint_kernel": 13,
})


def adjoint_case(device):
    """Frozen flow and state of the adjoint workload on ``device``."""
    import torch

    from gm1_b200.adjoint import FrozenFlow
    from gm1_b200.moist_step import MoistStepConfig, NativeMoistLargeStep, upload, weisman_klemp_initial_state
    from gm1_b200.scalar_rk import moisture_weps_f64, theta_weps_f64

    g = ADJOINT_GRID
    cfg = MoistStepConfig(**g)
    host, metrics = weisman_klemp_initial_state(cfg, **ADJOINT_INIT)
    model = NativeMoistLargeStep(cfg, upload(host, device), upload(metrics, device))
    for _ in range(ADJOINT_SPINUP):
        model.step()
    model.check()
    s, m = model.s, model.m
    ni, nj, nk = g["ni"], g["nj"], g["nk"]
    fields = {n: s[n].clone() for n in ("rru", "rrv", "rrw", "divx", "prs")}
    fields.update({n: m[n].clone() for n in ("c1", "c2", "rr0", "gz")})
    fields["th0"], fields["pi0"] = s["th0_3d"].clone(), s["pi0_3d"].clone()
    fields["pp3d"] = s["pp3d"][1:nk + 1, 1:nj + 1, 1:ni + 1].contiguous()
    flow = FrozenFlow(ni, nj, nk, g["dx"], g["dy"], g["dz"], theta_weps_f64(), fields)
    state = (s["th3d"].clone(), s["q3d"][0].clone(), s["q3d"][1].clone(), s["q3d"][2].clone())
    weps = {"th3d": theta_weps_f64(), "qv": moisture_weps_f64(0), "qc": moisture_weps_f64(1),
            "qr": moisture_weps_f64(2)}
    rho0 = m["rho0_3d"].clone()
    weights = (torch.zeros_like(rho0), torch.zeros_like(rho0), rho0, rho0)
    model.close()
    return flow, state, weps, weights


def adjoint_cpu_rate(seconds_target: float, threads: int) -> tuple[float, str]:
    """The binary64 restatement's gradient (torch autograd on the host
    cores) on a 32x32x48 sub-block of the workload's grid with a synthetic
    frozen flow, one large step per gradient."""
    import numpy as np
    import torch

    from oracle import adjoint_f64 as f64

    torch.set_num_threads(threads)
    ni, nj, nk = 32, 32, ADJOINT_GRID["nk"]
    rng = np.random.default_rng(4)
    t = lambda a: torch.from_numpy(np.asarray(a, np.float64))  # noqa: E731
    fr = {"rru": t(rng.uniform(-5, 15, (nk + 2, nj + 6, ni + 7))), "rrv": t(rng.uniform(-5, 15, (nk + 2, nj + 7, ni + 6))),
          "rrw": t(rng.uniform(-1, 1, (nk + 3, nj + 6, ni + 6))), "c1": t(np.full((nk + 1, nj, ni), 0.5)),
          "c2": t(np.full((nk + 1, nj, ni), 0.5)), "rr0": t(np.ones((nk, nj, ni))), "gz": t(np.ones((nj, ni))),
          "divx": t(np.zeros((nk, nj, ni))), "th0": t(np.full((nk, nj, ni), 300.0)),
          "pi0": t(np.full((nk, nj, ni), 0.95)), "pp3d": t(np.zeros((nk, nj, ni))),
          "prs": t(np.full((nk, nj, ni), 8.5e4))}
    state = {"th3d": t(rng.uniform(-1, 1, (nk, nj, ni))), "qv": t(rng.uniform(0.005, 0.015, (nk, nj, ni))),
             "qc": t(rng.uniform(0, 2e-3, (nk, nj, ni))), "qr": t(rng.uniform(0, 2e-3, (nk, nj, ni)))}
    kw = dict(ni=ni, nj=nj, nk=nk, dt=ADJOINT_GRID["dt"], dx=ADJOINT_GRID["dx"], dy=ADJOINT_GRID["dy"],
              dz=ADJOINT_GRID["dz"], weps=1e-6, steps=1)
    n, t0 = 0, time.perf_counter()
    while True:
        x = {k: v.clone().requires_grad_(True) for k, v in state.items()}
        out = f64.warm_rain_transport(x, fr, **kw)
        torch.autograd.grad((out["qc"] + out["qr"]).sum(), list(x.values()))
        n += 1
        dt = time.perf_counter() - t0
        if dt >= seconds_target or n >= 20:
            break
    return ni * nj * nk * n / dt, f"{n} one-step gradients of a {ni}x{nj}x{nk} sub-block in {dt:.2f} s"


def run_reference_adjoint(args) -> None:
    """The reference has no adjoint: its arm times the binary64 restatement
    of the same composition (oracle/adjoint_f64.py) on the host cores."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    threads = os.cpu_count() or 1
    value, sample = adjoint_cpu_rate(max(5.0, 2.0 * args.steps), threads)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "dtype": "f64",
        "config": {"workload": ADJOINT_NAME, "device": "host CPU", "note": "the reference has no adjoint"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


ADJOINT_NAME = ("adjoint of the warm-rain transport (theta', qv, qc, qr: RK3 WENO5 transport by frozen mass fluxes, "
                "collection, single-pass satadj) about a Weisman-Klemp supercell (cloudy bubble core) spun up 60 large "
                "steps (300 s) on 96x96x48 "
                "(dx=dy=1 km, dz=300 m, dt=5 s); J = sum(rho0 (qc + qr)) at the window's end")


def run_adjoint(args) -> None:
    """Forward sweep storing each large-step boundary, then the reverse sweep
    (recompute one step from its checkpoint, pull the adjoint back through
    the adjoint kernels), every step timed alone with L2 flushed before it."""
    import torch
    import torch.distributed as dist

    from gm1_b200 import _native
    from gm1_b200.adjoint import StepGraphs, WarmRainTransport
    from gm1_b200.autotune import Autotuner

    rank, world, local, device, barrier, max_over_ranks = _dist_setup()
    flow, state0, weps, weights = adjoint_case(device)
    tuner = Autotuner()
    model = WarmRainTransport(flow, ADJOINT_GRID["dt"], weps=weps, checkpoint=True, tuner=tuner)
    cells = flow.ni * flow.nj * flow.nk
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    model.gradient(state0, weights, args.warmup)
    graphs = StepGraphs(model, state0)
    graphs.gradient(state0, weights, args.warmup)
    torch.cuda.synchronize(device)

    x0, w0 = StepGraphs.stack(state0), StepGraphs.stack(weights)
    # the window's checkpoint store, laid out once (64 words per cell-step)
    store = graphs.store(args.steps)

    def sweep(k: int, fwd_ev, rev_ev):
        inputs, saved = [x0], []
        for q in range(k):
            flush.zero_()
            fwd_ev[q][0].record()
            saved.append(graphs.forward(inputs[-1], store[q]))
            fwd_ev[q][1].record()
            inputs.append(saved[-1][:4])
        adj = w0
        for q in reversed(range(k)):
            flush.zero_()
            rev_ev[q][0].record()
            adj = graphs.reverse(inputs[q], saved[q], adj)
            rev_ev[q][1].record()
        return tuple(adj[q] for q in range(4))

    def plain_forward(k: int, ev_):
        cur = x0
        for q in range(k):
            flush.zero_()
            ev_[q][0].record()
            cur = graphs.step(cur)
            ev_[q][1].record()

    ev = lambda: [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))  # noqa: E731
                  for _ in range(args.steps)]
    fwd_ev, rev_ev, plain_ev = ev(), ev(), ev()
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    grads = sweep(args.steps, fwd_ev, rev_ev)
    plain_forward(args.steps, plain_ev)
    barrier()
    clocks = sampler.stop()
    t_save = max_over_ranks(sum(a.elapsed_time(b) for a, b in fwd_ev))
    t_rev = max_over_ranks(sum(a.elapsed_time(b) for a, b in rev_ev))
    t_fwd = max_over_ranks(sum(a.elapsed_time(b) for a, b in plain_ev))
    t_adj = t_save + t_rev
    value = world * cells * args.steps / (t_adj * 1e-3)
    # the same window eagerly through autograd and torch.utils.checkpoint
    _, ref = model.gradient(state0, weights, args.steps)
    rel = {n: float((a.double() - b.double()).norm() / max(float(b.double().norm()), 1e-300))
           for n, a, b in zip(("th3d", "qv", "qc", "qr"), grads, ref)}
    finite = {n: bool(torch.isfinite(a).all()) for n, a in zip(("th3d", "qv", "qc", "qr"), grads)}
    finite_ref = {n: bool(torch.isfinite(b).all()) for n, b in zip(("th3d", "qv", "qc", "qr"), ref)}
    norms = {n: float(a.double().norm()) for n, a in zip(("th3d", "qv", "qc", "qr"), grads)}
    cloudy = int((state0[2] > 0).sum())

    # per-kernel device time of one stage-saving step and its reverse
    # (launch profiler, eager launches)
    from gm1_b200.adjoint import StageCheckpointedAdjoint

    sc = StageCheckpointedAdjoint(model)
    _native.profiler_enable(True)
    _, stages = sc.forward(state0)
    sc.reverse(stages, weights)
    torch.cuda.synchronize(device)
    _native.profiler_enable(False)
    stats = _native.profiler_collect()
    del stages
    launches = sum(x["launches"] for x in stats)
    peak, peak_kind = load_peaks()
    roofline = _kernel_roofline(stats, cells, peak, peak_kind)
    tot = sum(x["total_ms"] for x in stats)
    kernel_share = {x["name"]: round(x["total_ms"] / tot, 4) for x in stats[:12]}

    # e2e: the initial state in from pinned host memory and the gradient out,
    # around the whole gradient call
    pinned_in = [t.cpu().pin_memory() for t in state0]
    pinned_out = [torch.empty_like(t) for t in pinned_in]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    flush.zero_()
    e0.record()
    dev_in = tuple(t.to(device, non_blocking=True) for t in pinned_in)
    g = graphs.gradient(dev_in, weights, args.steps, store)
    for o, x in zip(pinned_out, g):
        o.copy_(x, non_blocking=True)
    e1.record()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = world * cells * args.steps / (e2e_ms * 1e-3)
    h2d = sum(t.numel() * 4 for t in pinned_in)
    del graphs
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, sample = adjoint_cpu_rate(10.0, threads)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": sample + " (the binary64 torch restatement of the same composition, autograd)"}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_adj / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic (seeded Weisman-Klemp start, numpy default_rng({ADJOINT_INIT['seed']}), spun up "
                f"{ADJOINT_SPINUP} steps by the moist model)",
        "config": {"workload": ADJOINT_NAME, "mode": "adjoint", "cells": cells,
                   "checkpoints": "every RK-stage boundary (the forward sweep keeps each scalar's stage states; "
                                  "the reverse rebuilds only each stage's open-filled carrier)",
                   "cuda_graphs": "plain step, stage-saving step and one-step reverse each replayed from one graph",
                   "checkpoint_store_bytes": store.numel() * 4,
                   "t_adj": "forward sweep with stage saves + reverse sweep; t_fwd: the plain forward step",
                   "levels_per_chunk": {"fifth_order": model.chunk[1], "weno5": model.chunk[3]},
                   "autotune_ms": tuner.table,
                   "t_fwd_ms_per_step": t_fwd / args.steps, "t_forward_sweep_ms_per_step": t_save / args.steps,
                   "t_reverse_sweep_ms_per_step": t_rev / args.steps,
                   "t_adj_over_t_fwd": t_adj / t_fwd, "target_t_adj_over_t_fwd": 3.0,
                   "relative_l2_vs_autograd_checkpoint_path": rel, "gradient_finite": finite,
                   "autograd_gradient_finite": finite_ref, "gradient_l2_norms": norms,
                   "cloudy_cells_at_start": cloudy,
                   "l2": "flushed before every timed large step, forward and reverse (256 MiB write, outside the "
                         "event pair)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single domain"},
        "step_roofline": {"bytes_per_cell_update": 4 * ADJOINT_WORDS,
                          "achieved_gbs": 4 * ADJOINT_WORDS * value / world / 1e9,
                          "frac": 4 * ADJOINT_WORDS * value / world / 1e9 / peak},
        "roofline": roofline, "kernel_share": kernel_share,
        "gpu_launches": int(launches * args.steps),
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": h2d // args.steps},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=("c3", "moist-c2", "dry", "ensemble", "adjoint"), default="c3")
    ap.add_argument("--members", type=int, default=64, help="ensemble members (--workload ensemble)")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = {"c3": 20, "moist-c2": 20, "ensemble": 10, "adjoint": 120}.get(args.workload, 2000)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        if args.workload == "adjoint":
            run_reference_adjoint(args)
            return
        (run_reference if args.workload == "dry" else run_reference_moist)(args)
        return
    if args.workload == "adjoint":
        run_adjoint(args)
        return
    if args.workload in MOIST_WORKLOADS:
        run_moist(args)
        return
    if args.workload == "ensemble":
        run_ensemble(args)
        return

    import torch
    import torch.distributed as dist

    from gm1_b200 import _native
    from gm1_b200.initial_state import DRY_BUBBLE_64, dry_periodic_state
    from gm1_b200.periodic import launch_cuda_psolver3_trajectory, to_device

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)

    c = DRY_BUBBLE_64
    host = dry_periodic_state(c)
    dev = to_device(host, device)
    # barrier status words are read once after the timed region, not per step
    p = dict(ni=c.ni, nj=c.nj, nk=c.nk, steps=1, dt=c.dt, nsound=c.nsound, dx=c.dx, dy=c.dy, dz=c.dz,
             scratch_outputs=False, check_status=False)
    stream = torch.cuda.Stream(device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    def barrier():
        torch.cuda.synchronize(device)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(device)

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            launch_cuda_psolver3_trajectory(dev, stream=stream, **p)
        stream.synchronize()
        graph = torch.cuda.CUDAGraph()
        try:
            with torch.cuda.graph(graph, stream=stream):
                captured = launch_cuda_psolver3_trajectory(dev, stream=stream, **p)
            use_graph = True
        except Exception as exc:  # noqa: BLE001 - capture refused: time direct launches
            print(f"CUDA graph capture failed ({exc}); timing direct launches", file=sys.stderr)
            torch.cuda.synchronize(device)
            use_graph = False

        def step() -> None:
            if use_graph:
                graph.replay()
            else:
                launch_cuda_psolver3_trajectory(dev, stream=stream, **p)

        for _ in range(args.warmup):
            step()
        stream.synchronize()

    # ---- timed region: K graph replays, L2 flushed before each ----------
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    with torch.cuda.stream(stream):
        for q in range(args.steps):
            flush.zero_()
            starts[q].record(stream)
            step()
            ends[q].record(stream)
    barrier()
    clocks = sampler.stop()
    if use_graph:
        captured.check()  # raises if a persistent stage's grid barrier gave up
    local_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    total_ms = max_over_ranks(local_ms)
    ms_per_step = total_ms / args.steps
    value = world * c.cells * args.steps / (total_ms * 1e-3)

    # ---- per-kernel device time (same steps, no graph, profiler on) ------
    _native.profiler_enable(True)
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()
            launch_cuda_psolver3_trajectory(dev, stream=stream, **p)
    stream.synchronize()
    _native.profiler_enable(False)
    stats = _native.profiler_collect()
    launches_per_step = sum(s["launches"] for s in stats) / args.steps
    top = stats[0]
    avg_ms = top["total_ms"] / top["launches"]
    alg_bytes = KERNEL_WORDS_PER_CELL[top["name"]] * 4 * c.cells
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (avg_ms * 1e-3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "traffic_per_launch.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get("dry", {}).get(top["name"])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": top["name"], "avg_launch_ms": avg_ms,
                "alg_bytes_per_launch": alg_bytes, "peak_source": f"{peak_kind} hbm_gbs"}
    kernel_share = {s["name"]: round(s["total_ms"] / sum(x["total_ms"] for x in stats), 4) for s in stats}

    # ---- e2e through the public API with pinned host buffers -------------
    pinned = {n: torch.from_numpy(host[n]).pin_memory() for n in PROGNOSTIC}
    h2d = sum(t.numel() * 4 for t in pinned.values())
    e_start = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_end = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    pe = dict(p)
    barrier()
    with torch.cuda.stream(stream):
        for q in range(args.steps):
            flush.zero_()
            e_start[q].record(stream)
            for n, t in pinned.items():
                dev[n].copy_(t, non_blocking=True)
            launch_cuda_psolver3_trajectory(dev, stream=stream, **pe)
            for n, t in pinned.items():
                t.copy_(dev[n], non_blocking=True)
            e_end[q].record(stream)
    barrier()
    e2e_ms = max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(e_start, e_end)))
    e2e_value = world * c.cells * args.steps / (e2e_ms * 1e-3)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_step_rate(3, 10.0, os.cpu_count() or 1)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded dry warm bubble, numpy default_rng(1) noise)",
        "config": {
            "workload": WORKLOAD,
            "mode": "fwd",
            "cells": c.cells,
            "large_steps_per_timed_step": 1,
            "acoustic_small_steps_per_step": 11,
            "l2": "flushed before every timed step (256 MiB write, outside the event pair)",
            "cuda_graph": use_graph,
            "parallelism": f"replicas x{world}" if world > 1 else "single domain",
        },
        "step_roofline": {"bytes_per_cell_update": STEP_BYTES_PER_CELL,
                          "achieved_gbs": STEP_BYTES_PER_CELL * value / world / 1e9,
                          "frac": STEP_BYTES_PER_CELL * value / world / 1e9 / peak},
        "roofline": roofline,
        "kernel_share": kernel_share,
        "gpu_launches": int(round(launches_per_step * args.steps)),
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
