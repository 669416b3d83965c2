"""Print each float32 prognostic field's error against the FP64 run of the
same operators, for the GPU step and for the binary32 oracle, as a markdown
table (needs a CUDA device):

    python -m tests.fp64_report [--quick]

Cases: configuration 2 at its full 256x256x80 size after one large step (the
benchmark's seeded Weisman-Klemp start: +3 K bubble of 10 km x 1.5 km at
1.5 km, U(+-0.1 K) noise, seed 2), and the 80-level stretched supercell
column of configuration 3 on a 128x128 plane after 1 and 20 large steps
(bubble 3 km x 1.5 km), also with the closure's held tendencies (SGS stress,
scalar diffusion, Rayleigh damping, dissipative heating).  Each cell of the table is "GPU / oracle", the
largest |error| divided by the field's largest |value| in the FP64 run.
"""

from __future__ import annotations

import argparse
import os

from gm1_b200.moist_step import (SUPERCELL_STRETCHED_COLUMN, MoistLargeStep, MoistStepConfig, upload,
                                 weisman_klemp_initial_state)
from tests.fp64_common import fp64_errors, table_header, table_rows


def _gpu(cfg, host, metrics):
    return MoistLargeStep(cfg, upload(host), upload(metrics))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true", help="reduced grids (a smoke run of the report)")
    args = ap.parse_args()
    threads = os.cpu_count() or 1
    c2 = (64, 64, 80) if args.quick else (256, 256, 80)
    c3 = (48, 40, 80) if args.quick else (128, 128, 80)
    cases = [
        (f"C2 {c2[0]}x{c2[1]}x{c2[2]}", MoistStepConfig(*c2, 1000.0, 1000.0, 250.0, 5.0, 10),
         dict(seed=2, bubble_k=3.0, noise_k=0.1, bubble_radius_m=(10000.0, 1500.0), bubble_center_z_m=1500.0), (1,)),
        (f"C3 column {c3[0]}x{c3[1]}x{c3[2]}",
         MoistStepConfig(*c3, 100.0, 100.0, 100.0, 0.6, 8, column=SUPERCELL_STRETCHED_COLUMN),
         dict(seed=2, bubble_k=3.0, noise_k=0.1, bubble_radius_m=(3000.0, 1500.0), bubble_center_z_m=1500.0),
         (1, 20)),
        (f"C3 column {c3[0]}x{c3[1]}x{c3[2]}, held closure",
         MoistStepConfig(*c3, 100.0, 100.0, 100.0, 0.6, 8, column=SUPERCELL_STRETCHED_COLUMN, sgs_diffusion=True,
                         rayleigh=True, dissipative_heating=True),
         dict(seed=2, bubble_k=3.0, noise_k=0.1, bubble_radius_m=(3000.0, 1500.0), bubble_center_z_m=1500.0),
         (1, 20)),
    ]
    lines = table_header()
    for label, cfg, init, steps in cases:
        host, metrics = weisman_klemp_initial_state(cfg, **init)
        lines += table_rows(label, fp64_errors(cfg, host, metrics, steps, _gpu, threads=threads))
    print("\n".join(lines), flush=True)


if __name__ == "__main__":
    main()
