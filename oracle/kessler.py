"""ctypes driver of the Kessler oracle (kessler_oracle.c) - TEST
INFRASTRUCTURE ONLY.  Mirrors cpu_gm1_kessler_driver_inplace
(src/cm1core/cuda_gm1_kessler_driver.py:431) for efall = 0."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)
_D = ctypes.POINTER(ctypes.c_double)
_U = ctypes.POINTER(ctypes.c_uint32)

FLOAT_NAMES = ("ruh", "rvh", "rmh", "mh", "pi0", "th0", "rr", "rho", "pp3d", "th3d", "prs", "qv", "qc", "qr",
               "fall_velocity", "rain", "prate")


class KesslerArrays(ctypes.Structure):
    _fields_ = [(n, _F) for n in FLOAT_NAMES] + [("asq", _D), ("qbudget", _D), ("satadj_iterations", _U)]


def _lib():
    lib = load()
    if not getattr(lib, "_kessler_ready", False):
        i, f = ctypes.c_int, C_REAL
        lib.oracle_kessler_driver.argtypes = [ctypes.POINTER(KesslerArrays), i, i, i, f, f, f, f, i,
                                              ctypes.POINTER(ctypes.c_int32)]
        lib.oracle_kessler_driver.restype = i
        lib._kessler_ready = True
    return lib


def kessler_driver(arrays, *, ni, nj, nk, dx, dy, dz, dt, eqtset, iterations=None, nfall=None) -> int:
    """Run in place; returns the largest fallout sub-step count (raises on
    satadj non-convergence, as the twin does)."""
    s = KesslerArrays()
    for n in FLOAT_NAMES:
        a = arrays[n]
        assert a.dtype == REAL and a.flags.c_contiguous
        setattr(s, n, a.ctypes.data_as(_F))
    for n in ("asq", "qbudget"):
        assert arrays[n].dtype == np.float64
        setattr(s, n, arrays[n].ctypes.data_as(_D))
    if iterations is not None:
        s.satadj_iterations = iterations.ctypes.data_as(_U)
    nf = nfall.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) if nfall is not None else None
    r = _lib().oracle_kessler_driver(ctypes.byref(s), ni, nj, nk, dx, dy, dz, dt, eqtset, nf)
    if r == -1:
        raise ValueError("invalid Kessler arguments")
    if r < -100:
        raise RuntimeError(f"Kessler satadj failed to converge in 100 iterations ({-r - 100} cells)")
    return r


HELD_NAMES = ("qpten", "qtten", "qvten", "qcten")


def dry_mass(rho, ruh, rvh, rmh, *, ni, nj, nk) -> float:
    """cpu_initial_dry_mass (src/cm1core/cuda_apmasscon.py:226) restated."""
    lib = load()
    if not getattr(lib, "_dry_mass_ready", False):
        lib.oracle_dry_mass.argtypes = [_F] * 4 + [ctypes.c_int] * 3
        lib.oracle_dry_mass.restype = ctypes.c_double
        lib._dry_mass_ready = True
    for a in (rho, ruh, rvh, rmh):
        assert a.dtype == REAL and a.flags.c_contiguous
    return float(lib.oracle_dry_mass(*(a.ctypes.data_as(_F) for a in (rho, ruh, rvh, rmh)), ni, nj, nk))


APMASSCON_NAMES = ("ruh", "rvh", "rmh", "pi0", "th0", "th3d", "qv", "pp3d", "prs", "rho")


def apmasscon(arrays, *, ni, nj, nk, mass1: float) -> np.ndarray:
    """cpu_apmasscon_inplace (src/cm1core/cuda_apmasscon.py:256) restated,
    in place; returns (mass2, Exner sum, binary64 correction, mass1)."""
    lib = load()
    if not getattr(lib, "_apmasscon_ready", False):
        lib.oracle_apmasscon.argtypes = [_F] * 11 + [ctypes.c_int] * 3 + [ctypes.c_double, _D]
        lib.oracle_apmasscon.restype = ctypes.c_int
        lib._apmasscon_ready = True
    for n in APMASSCON_NAMES:
        assert arrays[n].dtype == REAL and arrays[n].flags.c_contiguous, n
    diag = np.zeros(4, np.float64)
    r = lib.oracle_apmasscon(*(arrays[n].ctypes.data_as(_F) for n in APMASSCON_NAMES), None, ni, nj, nk,
                             float(mass1), diag.ctypes.data_as(_D))
    if r != 0:
        raise MemoryError("oracle_apmasscon")
    return diag


def kessler_large_step(arrays, held, *, ni, nj, nk, dx, dy, dz, dt, eqtset, nfall=None, mass1=None,
                       mass_diag=None) -> int:
    """cpu_gm1_kessler_large_step_inplace restated: held remove/snapshot,
    pre-physics EOS, (with mass1, a one-word float64 array: the dry-air mass
    correction), the driver, held recapture (in place)."""
    s = KesslerArrays()
    for n in FLOAT_NAMES:
        a = arrays[n]
        assert a.dtype == REAL and a.flags.c_contiguous
        setattr(s, n, a.ctypes.data_as(_F))
    for n in ("asq", "qbudget"):
        setattr(s, n, arrays[n].ctypes.data_as(_D))
    hp = (_F * 4)(*[held[n].ctypes.data_as(_F) for n in HELD_NAMES])
    lib = _lib()
    if not getattr(lib, "_kls_ready", False):
        lib.oracle_kessler_large_step.argtypes = [ctypes.POINTER(KesslerArrays), ctypes.POINTER(_F)] + \
            [ctypes.c_int] * 3 + [C_REAL] * 4 + [ctypes.c_int, ctypes.POINTER(ctypes.c_int32)]
        lib.oracle_kessler_large_step.restype = ctypes.c_int
        lib.oracle_kessler_large_step_apmasscon.argtypes = lib.oracle_kessler_large_step.argtypes + [_D, _D]
        lib.oracle_kessler_large_step_apmasscon.restype = ctypes.c_int
        lib._kls_ready = True
    nf = nfall.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) if nfall is not None else None
    if mass1 is None:
        r = lib.oracle_kessler_large_step(ctypes.byref(s), hp, ni, nj, nk, dx, dy, dz, dt, eqtset, nf)
    else:
        assert mass1.dtype == np.float64
        md = mass_diag if mass_diag is not None else np.zeros(4, np.float64)
        r = lib.oracle_kessler_large_step_apmasscon(ctypes.byref(s), hp, ni, nj, nk, dx, dy, dz, dt, eqtset, nf,
                                                    mass1.ctypes.data_as(_D), md.ctypes.data_as(_D))
    if r == -1:
        raise ValueError("invalid Kessler arguments")
    if r < -100:
        raise RuntimeError(f"Kessler satadj failed to converge in 100 iterations ({-r - 100} cells)")
    return r
