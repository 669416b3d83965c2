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


def kessler_large_step(arrays, held, *, ni, nj, nk, dx, dy, dz, dt, eqtset, nfall=None) -> int:
    """cpu_gm1_kessler_large_step_inplace restated: held remove/snapshot,
    pre-physics EOS, the driver, held recapture (in place)."""
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
        lib._kls_ready = True
    nf = nfall.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) if nfall is not None else None
    r = lib.oracle_kessler_large_step(ctypes.byref(s), hp, ni, nj, nk, dx, dy, dz, dt, eqtset, nf)
    if r == -1:
        raise ValueError("invalid Kessler arguments")
    if r < -100:
        raise RuntimeError(f"Kessler satadj failed to converge in 100 iterations ({-r - 100} cells)")
    return r
