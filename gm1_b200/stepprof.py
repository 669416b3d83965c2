"""Per-kernel device time of the composed moist step (the library's launch
profiler: CUDA events around every launch, one stream, no overlap):

    python -m gm1_b200.stepprof [--grid NI NJ NK] [--steps N] [--held] [--uniform]

The step is the C entry point's (gm1b_moist_large_step) on the seeded
Weisman-Klemp start of the 80-level stretched supercell column (20-500 m,
lid 20.8 km, dx = dy = 100 m, dt = 0.6 s, nsound = 8), or with
``--uniform`` of the uniform 250 m column (dx = dy = 1 km, dt = 5 s,
nsound = 10, the terrain operator family); ``--held`` turns on the
closure's held tendencies (SGS stress, scalar diffusion, upper Rayleigh
damping, dissipative heating).  One warm step, then ``--steps`` profiled
steps; prints each kernel's launches and milliseconds per step.
"""

from __future__ import annotations

import argparse
import dataclasses

import torch

from . import _native
from .moist_step import (SUPERCELL_STRETCHED_COLUMN, MoistStepConfig, NativeMoistLargeStep, upload,
                         weisman_klemp_initial_state)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", nargs=3, type=int, default=[640, 768, 80], metavar=("NI", "NJ", "NK"))
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--held", action="store_true", help="the closure's held tendencies on")
    ap.add_argument("--uniform", action="store_true", help="the uniform 250 m column")
    args = ap.parse_args()
    ni, nj, nk = args.grid
    if args.uniform:
        cfg = MoistStepConfig(ni, nj, nk, 1000.0, 1000.0, 250.0, 5.0, 10)
    else:
        cfg = MoistStepConfig(ni, nj, nk, 100.0, 100.0, 100.0, 0.6, 8, column=SUPERCELL_STRETCHED_COLUMN)
    if args.held:
        cfg = dataclasses.replace(cfg, sgs_diffusion=True, rayleigh=True, dissipative_heating=True)
    host, metrics = weisman_klemp_initial_state(cfg, seed=2, bubble_k=3.0, noise_k=0.1,
                                                bubble_radius_m=(10000.0, 1500.0), bubble_center_z_m=1500.0)
    dev = torch.device("cuda:0")
    st = torch.cuda.Stream(dev)
    with torch.cuda.stream(st):
        model = NativeMoistLargeStep(cfg, upload(host, dev), upload(metrics, dev), stream=st, concurrent=False)
        model.step()
        st.synchronize()
        _native.profiler_enable(True)
        for _ in range(args.steps):
            model.step()
        st.synchronize()
        _native.profiler_enable(False)
    model.check()
    model.close()
    stats = _native.profiler_collect()
    total = sum(x["total_ms"] for x in stats)
    print(f"{ni}x{nj}x{nk}{' uniform' if args.uniform else ''}{' with the held closure' if args.held else ''}: "
          f"{total / args.steps:.2f} ms per step "
          f"(sum of launch times)")
    print(f"{'kernel':40s} {'launches/step':>14s} {'ms/step':>9s} {'ms/launch':>10s} {'share':>6s}")
    for x in stats:
        print(f"{x['name']:40s} {x['launches'] / args.steps:14.1f} {x['total_ms'] / args.steps:9.3f} "
              f"{x['total_ms'] / x['launches']:10.3f} {x['total_ms'] / total:6.3f}")


if __name__ == "__main__":
    main()
