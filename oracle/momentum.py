"""ctypes driver of the momentum-advection oracle (momentum_oracle.c) - TEST
INFRASTRUCTURE ONLY.  Mirrors cpu_terrain_open_momentum_advection5_inplace
(src/cm1core/cuda_momentum_advection5.py:753)."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)
NAMES = ("u3d", "uten", "rru", "v3d", "vten", "rrv", "w3d", "wten", "rrw", "uh", "vh", "rho0_3d", "rf0", "rrf0", "c2",
         "gz", "gzu", "gzv", "rgzu", "rgzv", "dzdx", "dzdy", "divx")


class MomArrays(ctypes.Structure):
    _fields_ = [(n, _F) for n in NAMES]


def _lib():
    lib = load()
    if not getattr(lib, "_mom_ready", False):
        lib.oracle_momentum_advection5.argtypes = [ctypes.c_int] * 3 + [ctypes.POINTER(MomArrays),
                                                                          ctypes.POINTER(ctypes.c_int)] + \
            [C_REAL] * 3
        lib.oracle_momentum_advection5.restype = ctypes.c_int
        lib._mom_ready = True
    return lib


def momentum_advection5(a, *, ni, nj, nk, dx, dy, dz, lateral_sides=(2, 2, 2, 2)) -> None:
    s = MomArrays()
    for n in NAMES:
        v = a[n]
        assert v.dtype == REAL and v.flags.c_contiguous, n
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


COLUMN_PROFILES = ("rho0p", "sigma", "sigmaf", "rds", "rdsf", "mh", "mf", "rr0")


def momentum_advection5_column(a, column, *, ni, nj, nk, dx, dy, lateral_sides=(2, 2, 2, 2), phase=3) -> None:
    """The operator on a stretched column.  ``column`` holds ``flat`` and the
    profiles: rho0p (padded base density), and sigma/sigmaf/rds/rdsf/ztop
    (terrain branch) or mh/mf/rr0/rdz (flat column)."""
    s = MomArrays()
    for n in NAMES:
        setattr(s, n, a[n].ctypes.data_as(_F))
    lib = _lib()
    if not getattr(lib, "_mom_column_ready", False):
        lib.oracle_momentum_advection5_column_phase.argtypes = (
            [ctypes.c_int] * 3 + [ctypes.POINTER(MomArrays), ctypes.POINTER(ctypes.c_int), C_REAL,
                                  C_REAL, ctypes.c_int, ctypes.c_int] + [_F] * 5 + [C_REAL] +
            [_F] * 3 + [C_REAL])
        lib.oracle_momentum_advection5_column_phase.restype = ctypes.c_int
        lib._mom_column_ready = True
    keep = {n: np.ascontiguousarray(column[n], dtype=REAL) for n in COLUMN_PROFILES if column.get(n) is not None}
    ptr = {n: (keep[n].ctypes.data_as(_F) if n in keep else None) for n in COLUMN_PROFILES}
    sides = (ctypes.c_int * 4)(*lateral_sides)
    rc = lib.oracle_momentum_advection5_column_phase(
        ni, nj, nk, ctypes.byref(s), sides, dx, dy, phase, 1 if column["flat"] else 0, ptr["rho0p"], ptr["sigma"],
        ptr["sigmaf"], ptr["rds"], ptr["rdsf"], float(column.get("ztop", 0.0)), ptr["mh"], ptr["mf"], ptr["rr0"],
        float(column.get("rdz", 0.0)))
    if rc != 0:
        raise ValueError("oracle_momentum_advection5_column_phase failed")
