"""Stated tolerance of the SGS/TKE parity tests.

The grid scale (dx dy dz)^0.33333333 goes through a float32 power, which
differs by a few ULPs between NumPy (the reference's twin), the C library
(the oracle) and CUDA (the product); every word derived from it (length
scale, Km, Kh, dissipation, TKE source) inherits that.  Words that never meet
the power (tk, the model constants, the lower face) are compared bit for bit;
the others must satisfy max |error| <= 1e-5 * max |field| and
RMS(error) <= 2e-6 * RMS(field); the clip count is exact.
"""

from __future__ import annotations

import numpy as np

MAX_ABS_REL = 1.0e-5
REL_RMS = 2.0e-6
EXACT = ("tk", "cme", "ce1", "ce2", "tkea")
CLOSE = ("grdscl", "rgrdscl", "lenscl", "dissten", "kmh", "kmv", "khh", "khv", "tketen", "csm")


def assert_sgs_close(want: dict, got: dict) -> None:
    for n in EXACT:
        assert np.array_equal(want[n].view(np.uint32), got[n].view(np.uint32)), n
    for n in CLOSE:
        w = want[n].astype(np.float64)
        g = got[n].astype(np.float64)
        scale = max(float(np.max(np.abs(w))), 1e-30)
        rms = max(float(np.sqrt(np.mean(w * w))), 1e-30)
        assert float(np.max(np.abs(w - g))) <= MAX_ABS_REL * scale, n
        assert float(np.sqrt(np.mean((w - g) ** 2))) <= REL_RMS * rms, n
