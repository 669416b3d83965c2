"""ctypes driver of the CM1 limits oracle (limits_oracle.c) - TEST
INFRASTRUCTURE ONLY.  Mirrors src/cm1core/gm1_runtime.py:249-302,458-489 and
src/cm1core/storm_diagnostics.py:195-297."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)
_D = ctypes.c_double


def _lib():
    lib = load()
    if not getattr(lib, "_limits_ready", False):
        lib.oracle_small_step_limit.argtypes = [_D, _D]
        lib.oracle_small_step_limit.restype = _D
        lib.oracle_diagnostic_substeps.argtypes = [_D, _D, _D]
        lib.oracle_diagnostic_substeps.restype = ctypes.c_int
        lib.oracle_advective_courant.argtypes = [_D] * 7
        lib.oracle_advective_courant.restype = _D
        f = C_REAL
        lib.oracle_courant_max.argtypes = [ctypes.c_int] * 3 + [_F] * 6 + [f, f, f, _F]
        lib.oracle_courant_max.restype = f
        lib._limits_ready = True
    return lib


def small_step_limit(dx: float, dy: float) -> float:
    return float(_lib().oracle_small_step_limit(dx, dy))


def diagnostic_substeps(dt: float, dx: float, dy: float) -> int:
    return int(_lib().oracle_diagnostic_substeps(dt, dx, dy))


def advective_courant(dt, dx, dy, dz, u, v, w) -> float:
    return float(_lib().oracle_advective_courant(dt, dx, dy, dz, u, v, w))


def courant_max(u, v, w, uh, vh, mh, dtdx, dtdy, dtdz) -> tuple[float, np.ndarray]:
    nk, nj, ni1 = u.shape
    arrs = [np.ascontiguousarray(a, dtype=REAL) for a in (u, v, w, uh, vh, mh)]
    level = np.zeros(nk, REAL)
    p = [a.ctypes.data_as(_F) for a in arrs]
    out = _lib().oracle_courant_max(ni1 - 1, nj, nk, *p, dtdx, dtdy, dtdz, level.ctypes.data_as(_F))
    return float(np.float32(out)), level
