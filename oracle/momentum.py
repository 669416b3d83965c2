"""ctypes driver of the momentum-advection oracle (momentum_oracle.c) - TEST
INFRASTRUCTURE ONLY.  Mirrors cpu_terrain_open_momentum_advection5_inplace
(src/cm1core/cuda_momentum_advection5.py:753)."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import load

_F = ctypes.POINTER(ctypes.c_float)
NAMES = ("u3d", "uten", "rru", "v3d", "vten", "rrv", "w3d", "wten", "rrw", "uh", "vh", "rho0_3d", "rf0", "rrf0", "c2",
         "gz", "gzu", "gzv", "rgzu", "rgzv", "dzdx", "dzdy", "divx")


class MomArrays(ctypes.Structure):
    _fields_ = [(n, _F) for n in NAMES]


def _lib():
    lib = load()
    if not getattr(lib, "_mom_ready", False):
        lib.oracle_momentum_advection5.argtypes = [ctypes.c_int] * 3 + [ctypes.POINTER(MomArrays),
                                                                          ctypes.POINTER(ctypes.c_int)] + \
            [ctypes.c_float] * 3
        lib.oracle_momentum_advection5.restype = ctypes.c_int
        lib._mom_ready = True
    return lib


def momentum_advection5(a, *, ni, nj, nk, dx, dy, dz, lateral_sides=(2, 2, 2, 2)) -> None:
    s = MomArrays()
    for n in NAMES:
        v = a[n]
        assert v.dtype == np.float32 and v.flags.c_contiguous, n
        setattr(s, n, v.ctypes.data_as(_F))
    sides = (ctypes.c_int * 4)(*lateral_sides)
    rc = _lib().oracle_momentum_advection5(ni, nj, nk, ctypes.byref(s), sides, dx, dy, dz)
    if rc != 0:
        raise ValueError(f"oracle_momentum_advection5 failed ({rc})")


def momentum_advection5_phase(a, *, ni, nj, nk, dx, dy, dz, lateral_sides=(2, 2, 2, 2), phase) -> None:
    """phase 1: mass fluxes and divx; 2: advu/advv/advw from them."""
    s = MomArrays()
    for n in NAMES:
        setattr(s, n, a[n].ctypes.data_as(_F))
    lib = _lib()
    if not getattr(lib, "_mom_phase_ready", False):
        lib.oracle_momentum_advection5_phase.argtypes = list(lib.oracle_momentum_advection5.argtypes) + [ctypes.c_int]
        lib.oracle_momentum_advection5_phase.restype = ctypes.c_int
        lib._mom_phase_ready = True
    sides = (ctypes.c_int * 4)(*lateral_sides)
    if lib.oracle_momentum_advection5_phase(ni, nj, nk, ctypes.byref(s), sides, dx, dy, dz, phase) != 0:
        raise ValueError("oracle_momentum_advection5_phase failed")
