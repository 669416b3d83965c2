"""Per-field error measures of a composed moist step against the oracle's
composition.

Each prognostic field is compared on its own scale: the largest magnitude of
that field in the oracle's state (u, v and w each their own; theta' and pi'
their perturbation fields; qv, qc and qr each their own species; TKE).  The
reported pair is (max |gpu - oracle| / scale, RMS(gpu - oracle) / scale).
"""

from __future__ import annotations

import numpy as np

FIELDS = ("u3d", "v3d", "w3d", "th3d", "pp3d", "qv", "qc", "qr", "tke3d")

# Bars (max |err| / scale, RMS / scale), about ten times the largest error
# measured on a B200 over the composed-step tests of both column families.
# After 1 and 3 steps the words differ only by the ulps that powf/expf/sqrtf
# (Kessler, the TKE closure) round differently on CUDA and in the C library,
# carried through the step; qc, whose saturation adjustment switches on a
# threshold, is the widest.
SHORT_BARS = {"u3d": (5.0e-5, 2.0e-6), "v3d": (1.0e-4, 3.0e-6), "w3d": (3.0e-4, 7.0e-6), "th3d": (8.0e-4, 2.0e-5),
              "pp3d": (1.0e-3, 3.0e-5), "qv": (3.0e-5, 4.0e-7), "qc": (2.0e-2, 3.0e-4), "qr": (7.0e-6, 2.0e-7),
              "tke3d": (3.0e-4, 7.0e-6)}
# Over 60 steps of a convective start the ulp differences grow as the flow
# does and branch switches (saturation, TKE clipping, upwind choices) flip
# single cells; long runs are judged against the FP64 run of the same
# operators (tests/fp64_common.py: check_long_run), where the binary32
# oracle's own error shows how far the float32 rounding carries.


def _host(x):
    return x.cpu().numpy() if hasattr(x, "cpu") else x


def _field(s, name):
    if name in ("qv", "qc", "qr"):
        return _host(s["q3d"])[("qv", "qc", "qr").index(name)]
    return _host(s[name])


def field_errors(gpu_state, ref_state) -> dict[str, tuple[float, float]]:
    out = {}
    for n in FIELDS:
        g, r = _field(gpu_state, n).astype(np.float64), _field(ref_state, n).astype(np.float64)
        d = g - r
        scale = float(np.max(np.abs(r))) or 1.0
        out[n] = (float(np.max(np.abs(d))) / scale, float(np.sqrt(np.mean(d * d))) / scale)
    return out


def format_errors(err) -> str:
    return " ".join(f"{n}={a:.1e}/{b:.1e}" for n, (a, b) in err.items())


def check_errors(err, bars: dict[str, tuple[float, float]], what: str) -> None:
    bad = {n: e for n, e in err.items() if not (e[0] <= bars[n][0] and e[1] <= bars[n][1])}
    assert not bad, f"{what}: {format_errors(bad)} above {({n: bars[n] for n in bad})}"


def worst(a, b):
    return {n: (max(a[n][0], b[n][0]), max(a[n][1], b[n][1])) for n in FIELDS}
