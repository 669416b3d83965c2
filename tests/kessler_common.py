"""Shared pieces of the Kessler parity tests: the stated tolerances.

The Kessler operator passes values through powf/expf, which differ by a few
ULPs between NumPy (the reference's twin), the C library (the oracle) and
CUDA (the product); the iterative saturation adjustment then carries those
ULPs into every thermodynamic word.  So:

* words that never meet a transcendental (the pdefq pass and its budget asq)
  are compared bit for bit;
* each field's error is measured against the scale of the full variable it
  perturbs (theta = th0 + th3d for th3d, pi = pi0 + pp3d for pp3d, total
  water qv + qc + qr for the mixing ratios, the field itself otherwise):
  max |error| / scale <= 2e-6 (about 16 float32 ULPs of the full variable)
  and RMS(error) / RMS(full variable) <= 1e-6;
* each FP64 budget agrees to a relative 1e-5 of its own magnitude;
* integer outputs (fallout sub-step counts, saturation-adjustment iteration
  counts) are equal.
"""

from __future__ import annotations

import numpy as np

MAX_ABS_REL = 2.0e-6
REL_RMS = 1.0e-6
BUDGET_RTOL = 1.0e-5
FIELDS = ("rho", "pp3d", "th3d", "prs", "qv", "qc", "qr", "fall_velocity", "rain", "prate")


def full_variable(name: str, fields: dict) -> np.ndarray:
    if name == "th3d":
        return fields["th0"].astype(np.float64) + fields["th3d"]
    if name == "pp3d":
        return fields["pi0"].astype(np.float64) + fields["pp3d"]
    if name in ("qv", "qc", "qr"):
        return fields["qv"].astype(np.float64) + fields["qc"] + np.maximum(fields["qr"], 0)
    return fields[name].astype(np.float64)


def field_errors(name: str, want: dict, got: dict) -> tuple[float, float]:
    err = want[name].astype(np.float64) - got[name].astype(np.float64)
    full = full_variable(name, want)
    scale = max(float(np.max(np.abs(full))), 1e-30)
    rms = max(float(np.sqrt(np.mean(full * full))), 1e-30)
    return float(np.max(np.abs(err))) / scale, float(np.sqrt(np.mean(err * err))) / rms


def assert_fields_close(want: dict, got: dict, names=FIELDS) -> dict:
    report = {}
    for n in names:
        ma, rr = field_errors(n, want, got)
        report[n] = (ma, rr)
        assert ma <= MAX_ABS_REL and rr <= REL_RMS, (n, ma, rr)
    return report


def assert_budgets_close(want: np.ndarray, got: np.ndarray) -> None:
    bound = BUDGET_RTOL * np.maximum(np.abs(want), 1.0)
    assert np.all(np.abs(want - got) <= bound), (want, got)
