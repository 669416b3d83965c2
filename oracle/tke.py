"""ctypes driver of the SGS/TKE oracle (tke_oracle.c) - TEST INFRASTRUCTURE
ONLY.  Mirrors cpu_sgs_tke_inplace (src/cm1core/cuda_sgs_tke.py:220)."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)
NAMES = ("ruh", "rvh", "rmf", "nm", "defv", "defh", "tkea", "tk", "grdscl", "rgrdscl", "lenscl", "dissten", "cme",
         "ce1", "ce2", "csm", "kmh", "kmv", "khh", "khv", "tketen")


class SgsTkeArrays(ctypes.Structure):
    _fields_ = [(n, _F) for n in NAMES]


def _lib():
    lib = load()
    if not getattr(lib, "_tke_ready", False):
        lib.oracle_sgs_tke.argtypes = [ctypes.POINTER(SgsTkeArrays), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       C_REAL, C_REAL, C_REAL]
        lib.oracle_sgs_tke.restype = ctypes.c_int
        lib.oracle_sgs_constants.argtypes = [_F]
        lib.oracle_sgs_constants.restype = None
        lib._tke_ready = True
    return lib


def sgs_tke(arrays, *, ni, nj, nk, dx, dy, dz) -> int:
    s = SgsTkeArrays()
    for n in NAMES:
        a = arrays[n]
        assert a.dtype == REAL and a.flags.c_contiguous
        setattr(s, n, a.ctypes.data_as(_F))
    return int(_lib().oracle_sgs_tke(ctypes.byref(s), ni, nj, nk, dx, dy, dz))


def sgs_constants() -> dict[str, float]:
    out = np.zeros(4, REAL)
    _lib().oracle_sgs_constants(out.ctypes.data_as(_F))
    return dict(zip(("cme", "ce1", "ce2", "csm"), (float(x) for x in out)))
