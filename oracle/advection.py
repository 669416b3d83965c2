"""ctypes driver of the padded-lane advection oracle (advection_oracle.c) -
TEST INFRASTRUCTURE ONLY.

Mirrors cpu_terrain_mass_flux5_inplace and cpu_scalar_advection5_inplace
(src/cm1core/cuda_advection5.py:271,440) on dictionaries of float32 arrays;
``lateral_obc`` adds the whole-domain lateral-side behaviour of the
reference's CUDA tendency kernel (0 = the twin's tile-local launch).
"""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)


class MassFluxArrays(ctypes.Structure):
    _fields_ = [(n, _F) for n in ("u3d", "v3d", "w3d", "rru", "rrv", "rrw", "rho0_3d", "rf0", "rgzu", "rgzv",
                                  "dzdx", "dzdy", "gz", "divx")]


class ScalarAdvArrays(ctypes.Structure):
    _fields_ = [(n, _F) for n in ("scalar", "rru", "rrv", "rrw", "c1", "c2", "rr0", "gz", "divx", "tendency",
                                  "flux_x", "flux_y", "flux_z")]


def _fill(struct, arrays):
    for name, _ in struct._fields_:
        a = arrays[name]
        if a.dtype != REAL or not a.flags.c_contiguous:
            raise ValueError(f"{name} must be C-contiguous float32")
        setattr(struct, name, a.ctypes.data_as(_F))
    return struct


def _lib():
    lib = load()
    if not getattr(lib, "_adv_ready", False):
        lib.oracle_terrain_mass_flux5.argtypes = [ctypes.POINTER(MassFluxArrays), ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, C_REAL, C_REAL, C_REAL]
        lib.oracle_terrain_mass_flux5.restype = None
        lib.oracle_scalar_advection5.argtypes = [ctypes.POINTER(ScalarAdvArrays), ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_int, C_REAL, C_REAL,
                                                 C_REAL, ctypes.c_double, ctypes.c_uint]
        lib.oracle_scalar_advection5.restype = None
        lib.oracle_scalar_advection5_column.argtypes = [ctypes.POINTER(ScalarAdvArrays), ctypes.c_int, ctypes.c_int,
                                                        ctypes.c_int, ctypes.c_int, C_REAL, C_REAL,
                                                        ctypes.c_double, ctypes.c_uint, ctypes.c_int, _F, _F,
                                                        C_REAL]
        lib.oracle_scalar_advection5_column.restype = None
        lib.oracle_weno5.argtypes = [C_REAL] * 5 + [ctypes.c_double]
        lib.oracle_weno5.restype = C_REAL
        lib._adv_ready = True
    return lib


def terrain_mass_flux5(arrays, *, ni, nj, nk, dx, dy, dz) -> None:
    s = _fill(MassFluxArrays(), arrays)
    _lib().oracle_terrain_mass_flux5(ctypes.byref(s), ni, nj, nk, dx, dy, dz)


def scalar_advection5(arrays, *, ni, nj, nk, nrk, dx, dy, dz, weps, wflag=True, lateral_obc=0) -> None:
    use_weno = 1 if (wflag and nrk == 3) else 0
    s = _fill(ScalarAdvArrays(), arrays)
    _lib().oracle_scalar_advection5(ctypes.byref(s), ni, nj, nk, use_weno, dx, dy, dz, weps, lateral_obc)


def scalar_advection5_column(arrays, *, ni, nj, nk, nrk, dx, dy, weps, flat, profile, rdz=0.0, wflag=True,
                             lateral_obc=0) -> None:
    """Stretched column: flat=False takes profile = rdsf (nk+3 words, CM1
    indexing), flat=True profile = mh (nk+2 words) with rdz."""
    use_weno = 1 if (wflag and nrk == 3) else 0
    s = _fill(ScalarAdvArrays(), arrays)
    prof = np.ascontiguousarray(profile, dtype=REAL)
    ptr = prof.ctypes.data_as(_F)
    _lib().oracle_scalar_advection5_column(ctypes.byref(s), ni, nj, nk, use_weno, dx, dy, weps, lateral_obc,
                                           2 if flat else 1, None if flat else ptr, ptr if flat else None, rdz)


def weno5(values, weps) -> float:
    return float(_lib().oracle_weno5(*[float(v) for v in values], float(weps)))
