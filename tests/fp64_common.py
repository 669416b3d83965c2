"""Each float32 prognostic field's error against the FP64 run of the same
operators (oracle/fp64_twin.py), for the GPU step and for the binary32
oracle side by side.

The FP64 run is the oracle's composition with every binary32 operation
evaluated in binary64, started from the same float32 words; its distance to a
float32 run is that run's rounding error.  Each field is measured on its own
scale (tests/moist_common.py: max |err| / max |field|, RMS / max |field|).
The GPU step passes when its error is of the size of the binary32 oracle's,
the reference algorithm's own float32 error: at most FP64_FACTOR times it,
plus FP64_FLOOR (of the field's scale) for fields the oracle reproduces to
the last few words.
"""

from __future__ import annotations

import numpy as np
import torch

from oracle.fp64_twin import run_fp64
from oracle.moist_composition import OracleMoistStep
from tests.moist_common import FIELDS, field_errors, format_errors

FP64_FACTOR = 4.0
FP64_FLOOR = (2.0e-6, 2.0e-7)
KEEP = ("u3d", "v3d", "w3d", "th3d", "pp3d", "q3d", "tke3d")


def fp64_errors(cfg, host: dict, metrics: dict, steps, make_gpu_step, threads: int | None = None):
    """{step: (gpu error, binary32-oracle error)} against the FP64 run, both
    per field as (max, RMS) on the field's own scale.  make_gpu_step(cfg,
    host, metrics) returns an object with .step() and .s (device state)."""
    steps = sorted(set(steps))
    last = steps[-1]
    h0 = {k: v.copy() for k, v in host.items()}
    m0 = {k: v.copy() for k, v in metrics.items()}
    f64 = run_fp64(cfg, h0, m0, last, snapshots=steps, threads=threads)
    dev = make_gpu_step(cfg, host, metrics)
    ref = OracleMoistStep(cfg, {k: v.copy() for k, v in host.items()}, {k: v.copy() for k, v in metrics.items()})
    out = {}
    for n in range(1, last + 1):
        dev.step()
        ref.step()
        if n in steps:
            torch.cuda.synchronize()
            gpu = {k: dev.s[k].cpu().numpy() for k in KEEP}
            out[n] = (field_errors(gpu, f64[n]), field_errors(ref.s, f64[n]))
    return out


def fp64_bars(oracle_err):
    return {n: (FP64_FACTOR * oracle_err[n][0] + FP64_FLOOR[0], FP64_FACTOR * oracle_err[n][1] + FP64_FLOOR[1])
            for n in FIELDS}


def table_rows(label: str, errs) -> list[str]:
    """Markdown rows: one per step, each field's GPU and oracle max error."""
    rows = []
    for step, (g, o) in sorted(errs.items()):
        cells = " | ".join(f"{g[n][0]:.1e} / {o[n][0]:.1e}" for n in FIELDS)
        rows.append(f"| {label} | {step} | {cells} |")
    return rows


def table_header() -> list[str]:
    return ["| case | step | " + " | ".join(FIELDS) + " |", "|---|---|" + "---|" * len(FIELDS)]


def describe(errs) -> str:
    return "; ".join(f"step {s}: gpu {format_errors(g)} | oracle {format_errors(o)}" for s, (g, o) in errs.items())


# Over a long run the two binary32 runs' own libm words keep entering: the
# Kessler rain terms and the equation-set-2 pressure pass through powf and
# expf in every cell every step, and CUDA documents its single-precision
# powf/expf to a few ulps where the C library's are within one, so the GPU's
# distance to the FP64 run may grow a few times faster than the oracle's
# (measured on the shallow column over 60 steps: rain 13x, theta RMS 2.4x).
LONG_RUN_FACTOR = 16.0


def check_long_run(cfg, host: dict, metrics: dict, make_gpu_step, steps: int = 60, every: int = 10,
                   what: str = "", factor: float = LONG_RUN_FACTOR) -> dict:
    """A long run's worst error against the FP64 run, GPU beside the binary32
    oracle: over the checkpoints every ``every`` steps, each field's largest
    GPU error (max and RMS on the field's scale) at most ``factor`` times the
    oracle's largest plus FP64_FLOOR.  Returns {step: (gpu, oracle)}."""
    from tests.moist_common import check_errors, worst

    errs = fp64_errors(cfg, host, metrics, tuple(range(every, steps + 1, every)), make_gpu_step)
    zero = {n: (0.0, 0.0) for n in FIELDS}
    gpu_w, ora_w = zero, zero
    for step, (g, o) in sorted(errs.items()):
        print(what, "after", step, "gpu vs fp64:", format_errors(g), "| oracle vs fp64:", format_errors(o))
        gpu_w, ora_w = worst(gpu_w, g), worst(ora_w, o)
    bars = {n: (factor * ora_w[n][0] + FP64_FLOOR[0], factor * ora_w[n][1] + FP64_FLOOR[1]) for n in FIELDS}
    check_errors(gpu_w, bars, f"{what} worst over {steps} steps against the FP64 run")
    return errs
