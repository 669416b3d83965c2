"""Per-operator device throughput on B200 (library profiling facility).

    python -m gm1_b200.opbench [--ops adv5 adv5-weno massflux calcdef moistnm courant tos tos-diag
                                      tos-stretched tos-flat moist]
                               [--grid 256 256 80] [--iters 20] [--nsound 10]

For each operator: seeded synthetic inputs of the given padded-lane grid
resident in HBM, a 256 MiB L2 flush before every launch, CUDA events around
each launch on the launching stream; prints one JSON line per operator with
cells/s, the average launch time, the algorithmic bytes per cell (every full
field read or written once; halos, stencil re-reads and 2-D metrics not
counted) and the fraction of the measured HBM copy bandwidth.
"""

from __future__ import annotations

import argparse
import json
from pathlib import Path

import numpy as np
import torch

from .advection import launch_cuda_scalar_advection5, launch_cuda_terrain_mass_flux5, padded_shapes

ROOT = Path(__file__).resolve().parents[1]

# words per cell
ALG_WORDS = {
    # in: scalar rru rrv rrw divx rr0 c1 c2; out: tendency
    "adv5": 9,
    "adv5-weno": 9,
    # in: u v w rho0 rf0; out: rru rrv rrw divx
    "massflux": 9,
    # in: u v w rho rf c1 c2 gx gy; out: defv defh
    "calcdef": 11,
    # in: c1 c2 mf prs pp3d th3d q3d(6); out: nm temperature qt thv qvci, mask (1 byte)
    "moistnm": 17.25,
    # in: u v w (one reduction)
    "courant": 3,
}


def moist_words(nsound: int) -> int:
    """Words per cell of one composed moist large step: 149 outside the
    acoustic loops plus 20 per small step over the three stages."""
    from .periodic import sound3_stage_schedule_f32  # noqa: PLC0415

    return 149 + 20 * sum(sound3_stage_schedule_f32(5.0, nsound, nrk)[0] for nrk in (1, 2, 3))


def tos_words(nloop: int) -> int:
    """Words per cell of one terrain/open acoustic stage: the prepare pass
    (in: ppx ppi ua va wa ppterm piadv c1 c2 rf0 rr0 thv; out: ppd pp3d rru
    rrv rrw u v w qk pk1 pk2 mm) and per small step the pressure gradient
    (in: ppd thv uten vten gxu gyv u v; out: u v) and the column pass (in: u
    v w pp3d qk pk1 pk2 mm ppten ppterm piadv rr0 rrf0 wten rru rrv rrw;
    out: w pp3d ppd rru rrv rrw)."""
    return 24 + 33 * nloop

_COMPACT: dict = {}
NSOUND = [10]
_CACHE: dict = {}


def compact_inputs(op: str, ni: int, nj: int, nk: int, device: torch.device) -> dict:
    """Seeded compact-layout inputs of the closure operators (built once)."""
    key = (op, ni, nj, nk)
    if key in _COMPACT:
        return _COMPACT[key]
    g = torch.Generator(device="cpu").manual_seed(3)

    def r(shape, lo, hi):
        return (torch.rand(shape, generator=g) * (hi - lo) + lo).to(device)

    cell, face = (nk, nj, ni), (nk + 1, nj, ni)
    if op == "calcdef":
        a = {"u3d": r((nk, nj, ni + 1), -10, 10), "v3d": r((nk, nj + 1, ni), -10, 10), "w3d": r(face, -2, 2),
             "rho": r(cell, 0.6, 1.2), "rf": r(face, 0.6, 1.2), "c1": r(face, 0.4, 0.6), "gz": r((nj, ni), 1, 1.02),
             "rgz": r((nj, ni), 0.98, 1), "gzu": r((nj, ni + 1), 1, 1.02), "rgzu": r((nj, ni + 1), 0.98, 1),
             "gzv": r((nj + 1, ni), 1, 1.02), "rgzv": r((nj + 1, ni), 0.98, 1), "gx": r(face, -1e-3, 1e-3),
             "gy": r(face, -1e-3, 1e-3), "defv": torch.empty(face, device=device),
             "defh": torch.empty(face, device=device)}
        a["c2"] = 1.0 - a["c1"]
    elif op == "moistnm":
        a = {"c1": r(face, 0.4, 0.6), "mf": r(face, 0.9, 1.1), "pi0": torch.linspace(1.0, 0.55, nk, device=device),
             "th0": torch.linspace(300.0, 380.0, nk, device=device), "prs": r(cell, 2e4, 1e5),
             "pp3d": r(cell, -1e-3, 1e-3), "th3d": r(cell, -2, 2), "q3d": r((6, nk, nj, ni), 0, 2e-3)}
        a["c2"] = 1.0 - a["c1"]
        for n in ("temperature", "qt", "thv", "qvci"):
            a[n] = torch.empty(cell, device=device)
        a["nm"] = torch.empty(face, device=device)
        a["saturation_mask"] = torch.empty(cell, dtype=torch.uint8, device=device)
    else:  # courant
        a = {"u": r((nk, nj, ni + 1), -30, 30), "v": r((nk, nj + 1, ni), -30, 30), "w": r((nk + 1, nj, ni), -5, 5),
             "uh": torch.ones(ni, device=device), "vh": torch.ones(nj, device=device),
             "mh": torch.ones(nk, device=device), "keys": torch.empty(nk, dtype=torch.int32, device=device),
             "out": torch.empty(1, device=device)}
    _COMPACT[key] = a
    return a


def tos_inputs(ni: int, nj: int, nk: int, device: torch.device, diag: bool) -> tuple[dict, dict]:
    """Seeded terrain/open acoustic-stage state and metrics (built once)."""
    key = ("tos", ni, nj, nk, diag)
    if key in _COMPACT:
        return _COMPACT[key]
    from .terrain_open import COLUMN_DIAGNOSTIC_NAMES, terrain_open_sound_shapes, terrain_static_shapes  # noqa: PLC0415

    g = torch.Generator(device=device).manual_seed(5)

    def r(shape, lo, hi):
        return torch.rand(shape, generator=g, device=device) * (hi - lo) + lo

    sh = terrain_open_sound_shapes(ni, nj, nk)
    a = {n: r(s, -0.5, 0.5) for n, s in sh.items()}
    for n in ("ppi", "pp3d", "ppx"):
        a[n] = r(sh[n], -2e-4, 2e-4)
    a["piadv"] = r(sh["piadv"], 0.89, 0.91)
    a["ppterm"] = a["piadv"] * 0.4
    a["thv"] = r(sh["thv"], 299.0, 331.0)
    a["ppten"] = r(sh["ppten"], -1e-6, 1e-6)
    for n, lo, hi in (("u3d", 4.0, 12.0), ("v3d", -6.0, 2.0), ("w3d", -0.5, 0.5)):
        a[n] = r(sh[n], lo, hi)
        a[n[0] + "a"] = a[n] + r(sh[n], -0.05, 0.05)
    for n in ("uten", "vten", "wten"):
        a[n] = r(sh[n], -2e-3, 2e-3)
    a["radbcw"], a["radbcs"] = r(sh["radbcw"], -25.0, 0.0), r(sh["radbcs"], -25.0, 0.0)
    a["radbce"], a["radbcn"] = r(sh["radbce"], 0.0, 25.0), r(sh["radbcn"], 0.0, 25.0)
    for n in ("uh", "vh", "ruf", "rvf"):
        a[n] = torch.ones(sh[n], device=device)
    if not diag:
        for n in COLUMN_DIAGNOSTIC_NAMES:
            a[n] = torch.zeros((1,), device=device)
    ms = terrain_static_shapes(ni=ni, nj=nj, nk=nk)
    m = {n: r(s, 0.95, 1.05) for n, s in ms.items()}
    m["c1"] = r(ms["c1"], 0.4, 0.6)
    m["c2"] = 1.0 - m["c1"]
    for n in ("dzdx", "dzdy"):
        m[n] = r(ms[n], -0.02, 0.02)
    for n in ("gx", "gxu", "gy", "gyv"):
        m[n] = r(ms[n], -0.005, 0.005)
    _COMPACT[key] = (a, m)
    return a, m


def hbm_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def synthetic_padded(ni: int, nj: int, nk: int, device: torch.device, seed: int = 0) -> dict[str, torch.Tensor]:
    g = torch.Generator(device=device).manual_seed(seed)
    sh = padded_shapes(ni, nj, nk)

    def u(shape, lo, hi):
        return (torch.rand(shape, generator=g, device=device) * (hi - lo) + lo).contiguous()

    a = {
        "scalar": u(sh["scalar"], 290.0, 310.0),
        "rru": u(sh["u"], -9.0, 9.0), "rrv": u(sh["v"], -9.0, 9.0), "rrw": u(sh["w"], -2.0, 2.0),
        "u3d": u(sh["u"], -12.0, 12.0), "v3d": u(sh["v"], -12.0, 12.0), "w3d": u(sh["w"], -3.0, 3.0),
        "c1": u(sh["face"], 0.3, 0.7), "rr0": u(sh["cell"], 0.8, 1.6), "rho0_3d": u(sh["cell"], 0.6, 1.2),
        "rf0": u(sh["face"], 0.6, 1.2), "divx": u(sh["cell"], -1e-3, 1e-3),
        "gz": u((nj, ni), 0.97, 1.03), "rgzu": u((nj, ni + 1), 0.95, 1.05), "rgzv": u((nj + 1, ni), 0.95, 1.05),
        "dzdx": u((nj, ni), -0.02, 0.02), "dzdy": u((nj, ni), -0.02, 0.02),
        "tendency": torch.zeros(sh["cell"], device=device),
        "mf_rru": torch.zeros(sh["u"], device=device), "mf_rrv": torch.zeros(sh["v"], device=device),
        "mf_rrw": torch.zeros(sh["w"], device=device), "mf_divx": torch.zeros(sh["cell"], device=device),
    }
    a["c2"] = 1.0 - a["c1"]
    return a


def run(op: str, a: dict[str, torch.Tensor], ni: int, nj: int, nk: int, stream: torch.cuda.Stream, chunk: int | None):
    if op in ("adv5", "adv5-weno"):
        launch_cuda_scalar_advection5(
            a["scalar"], {k: a[k] for k in ("rru", "rrv", "rrw")}, {k: a[k] for k in ("c1", "c2", "rr0", "gz")},
            a["divx"], a["tendency"], None, ni=ni, nj=nj, nk=nk, nrk=3 if op == "adv5-weno" else 1,
            dx=1000.0, dy=1000.0, dz=250.0, weps=1e-6, lateral_sides=(1, 1, 1, 1), write_fluxes=False,
            levels_per_chunk=chunk, stream=stream)
    elif op == "massflux":
        launch_cuda_terrain_mass_flux5(
            {"u3d": a["u3d"], "v3d": a["v3d"], "w3d": a["w3d"], "rru": a["mf_rru"], "rrv": a["mf_rrv"],
             "rrw": a["mf_rrw"]},
            {k: a[k] for k in ("rho0_3d", "rf0", "rgzu", "rgzv", "dzdx", "dzdy", "gz")}, a["mf_divx"],
            ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=250.0, stream=stream)
    elif op == "calcdef":
        from .closure import launch_cuda_terrain_deformation  # noqa: PLC0415

        c = compact_inputs(op, ni, nj, nk, a["u3d"].device)
        launch_cuda_terrain_deformation(c, ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=250.0, stream=stream)
    elif op == "moistnm":
        from .closure import launch_cuda_moist_nm  # noqa: PLC0415

        c = compact_inputs(op, ni, nj, nk, a["u3d"].device)
        launch_cuda_moist_nm(c, ni=ni, nj=nj, nk=nk, dz=250.0, stream=stream)
    elif op == "courant":
        from .limits import advective_courant_number  # noqa: PLC0415

        c = compact_inputs(op, ni, nj, nk, a["u3d"].device)
        advective_courant_number(u=c["u"], v=c["v"], w=c["w"], uh=c["uh"], vh=c["vh"], mh=c["mh"], dt_s=6.0,
                                 dx_m=1000.0, dy_m=1000.0, dz_m=250.0, level_keys=c["keys"], stream=stream,
                                 out=c["out"])
    elif op == "moist":
        key = ("moist", ni, nj, nk)
        if key not in _CACHE:
            from .moist_step import MoistLargeStep, MoistStepConfig, upload, weisman_klemp_initial_state  # noqa: PLC0415

            cfg = MoistStepConfig(ni, nj, nk, 1000.0, 1000.0, 250.0, 5.0, NSOUND[0])
            host, metrics = weisman_klemp_initial_state(cfg, seed=2, bubble_radius_m=(10000.0, 1500.0),
                                                        bubble_center_z_m=1500.0)
            dev = a["u3d"].device
            _CACHE[key] = MoistLargeStep(cfg, upload(host, dev), upload(metrics, dev), stream=stream)
        _CACHE[key].step()
    elif op in ("tos", "tos-diag"):
        from .terrain_open import compile_cuda_psolver3_terrain_open, launch_cuda_psolver3_terrain_open_stage  # noqa: PLC0415

        diag = op == "tos-diag"
        st, m = tos_inputs(ni, nj, nk, a["u3d"].device, diag)
        launch_cuda_psolver3_terrain_open_stage(
            st, m, ni=ni, nj=nj, nk=nk, nrk=3, dt=6.0, nsound=NSOUND[0], dx=1000.0, dy=1000.0, dz=250.0,
            compiled=compile_cuda_psolver3_terrain_open(retain_column_diagnostics=diag), stream=stream)
    elif op in ("tos-stretched", "tos-flat"):
        # the acoustic stage on the stretched column of the 640x768x80
        # supercell (stretch_z 1, 20 m at the ground to 500 m aloft, lid
        # 20.8 km): terrain branch or flat column, compact scratch
        from .momentum import StretchedMomentumColumn  # noqa: PLC0415
        from .terrain_open import (compile_cuda_psolver3_terrain_open,  # noqa: PLC0415
                                   launch_cuda_gm1_child_psolver3_open_stage)
        from .vertical import build_vertical_levels  # noqa: PLC0415

        dev = a["u3d"].device
        st, m = tos_inputs(ni, nj, nk, dev, False)
        key = (op, ni, nj, nk)
        if key not in _CACHE:
            if nk != 80:
                raise ValueError(f"{op} runs the nk = 80 stretched column")
            lv = build_vertical_levels(stretch_z=1, nk=80, dz_m=100.0, ztop_m=20800.0, str_bot_m=200.0,
                                       str_top_m=15800.0, dz_bot_m=20.0, dz_top_m=500.0)
            t = lambda x: torch.from_numpy(np.array(x, dtype=np.float32)).to(dev)  # noqa: E731
            m["rho0_padded"] = torch.ones((nk + 2, nj + 6, ni + 6), device=dev)
            _CACHE[key] = (StretchedMomentumColumn(True, None, mh=t(lv.mh), mf=t(lv.mf), rdz=0.01)
                           if op == "tos-flat" else
                           StretchedMomentumColumn(False, None, sigma=t(lv.sigma), sigmaf=t(lv.sigmaf), rds=t(lv.rds),
                                                   rdsf=t(lv.rdsf), ztop=lv.ztop_m))
        launch_cuda_gm1_child_psolver3_open_stage(
            st, m, ni=ni, nj=nj, nk=nk, nrk=3, dt=6.0, nsound=NSOUND[0], dx=1000.0, dy=1000.0, vertical=_CACHE[key],
            compiled=compile_cuda_psolver3_terrain_open(retain_column_diagnostics=False), stream=stream)
    else:
        raise ValueError(op)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ops", nargs="+", default=["adv5", "adv5-weno", "massflux"])
    ap.add_argument("--grid", nargs=3, type=int, default=[256, 256, 80], metavar=("NI", "NJ", "NK"))
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--chunk", type=int, default=None)
    ap.add_argument("--nsound", type=int, default=10, help="acoustic substeps of the terrain/open stage (nrk=3)")
    args = ap.parse_args()
    NSOUND[0] = args.nsound
    ni, nj, nk = args.grid
    device = torch.device("cuda", 0)
    a = synthetic_padded(ni, nj, nk, device)
    flush = torch.empty(256 * 1024 * 1024 // 4, device=device)
    stream = torch.cuda.Stream(device)
    peak, kind = hbm_peak()
    cells = ni * nj * nk
    for op in args.ops:
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                run(op, a, ni, nj, nk, stream, args.chunk)
            starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.iters)]
            ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.iters)]
            for q in range(args.iters):
                flush.zero_()
                starts[q].record(stream)
                run(op, a, ni, nj, nk, stream, args.chunk)
                ends[q].record(stream)
        stream.synchronize()
        ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / args.iters
        words = (tos_words(args.nsound) if op.startswith("tos")
                 else moist_words(args.nsound) if op == "moist" else ALG_WORDS[op])
        alg = words * 4 * cells
        gbs = alg / (ms * 1e-3) / 1e9
        print(json.dumps({"op": op, "grid": [ni, nj, nk], "cells": cells, "ms_per_launch": ms,
                          "cells_per_s": cells / (ms * 1e-3), "alg_bytes_per_cell": words * 4,
                          "achieved_gbs": gbs, "peak_gbs": peak, "frac": gbs / peak, "peak_source": kind,
                          "chunk": args.chunk}), flush=True)


if __name__ == "__main__":
    main()
