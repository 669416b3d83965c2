"""ctypes driver of the eqtset=2 cell oracle (rk_oracle.c) - TEST
INFRASTRUCTURE ONLY.  Mirrors cpu_eqtset2_cell_f32
(src/cm1core/cuda_moist_stage_bridge.py:62)."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)


def _lib():
    lib = load()
    if not getattr(lib, "_bridge_ready", False):
        f = C_REAL
        lib.oracle_eqtset2_cell.argtypes = [f, f, f, f, f, f, f, _F, _F]
        lib.oracle_eqtset2_cell.restype = None
        lib._bridge_ready = True
    return lib


def eqtset2_cell(th0, qv0, pi0, qc0, qi0, th3d, pp3d, q) -> np.ndarray:
    """(buoyancy, theta_rho, theta_term, pressure_term) of one cell."""
    qq = np.ascontiguousarray(q, dtype=REAL)
    out = np.zeros(4, REAL)
    _lib().oracle_eqtset2_cell(th0, qv0, pi0, qc0, qi0, th3d, pp3d, qq.ctypes.data_as(_F), out.ctypes.data_as(_F))
    return out


def eqtset2_stage_terms(*, ni, nj, nk, th0, qv0, pi0, th3d, q3d, pp3d, thv, ppterm, buoyancy, thterm, piadv) -> None:
    """The stage-terms pass over the padded lane (base profiles, zero base condensate)."""
    lib = _lib()
    if not getattr(lib, "_terms_ready", False):
        lib.oracle_eqtset2_stage_terms.argtypes = [ctypes.c_int] * 3 + [_F] * 11
        lib.oracle_eqtset2_stage_terms.restype = None
        lib._terms_ready = True
    ptrs = []
    for a in (th0, qv0, pi0, th3d, q3d, pp3d, thv, ppterm, buoyancy, thterm, piadv):
        assert a.dtype == REAL and a.flags.c_contiguous
        ptrs.append(a.ctypes.data_as(_F))
    lib.oracle_eqtset2_stage_terms(ni, nj, nk, *ptrs)
