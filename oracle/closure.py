"""ctypes driver of the closure-input oracle (closure_oracle.c) - TEST
INFRASTRUCTURE ONLY.  Mirrors cpu_terrain_deformation_inplace
(src/cm1core/cuda_terrain_deformation.py:234) and cpu_moist_nm_inplace
(src/cm1core/cuda_moist_nm.py:292)."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)

DEFORMATION_INPUTS = ("u3d", "v3d", "w3d", "rho", "rf", "c1", "c2", "gz", "rgz", "rgzu", "rgzv", "gx", "gy")
NM_INPUTS = ("c1", "c2", "mf", "pi0", "th0", "prs", "pp3d", "th3d", "q3d")
NM_OUTPUTS = ("nm", "temperature", "qt", "thv", "qvci")


def _lib():
    lib = load()
    if not getattr(lib, "_closure_ready", False):
        i, f = ctypes.c_int, C_REAL
        lib.oracle_calcdef.argtypes = [i, i, i] + [_F] * 13 + [f, f, f, _F, _F]
        lib.oracle_calcdef.restype = i
        lib.oracle_moist_nm.argtypes = [i, i, i] + [_F] * 9 + [f] + [_F] * 5 + [ctypes.c_void_p,
                                                                           ctypes.POINTER(ctypes.c_int64)]
        lib.oracle_moist_nm.restype = i
        lib.oracle_flat_calcdef.argtypes = [i, i, i] + [_F] * 9 + [f, f, f, _F, _F]
        lib.oracle_flat_calcdef.restype = i
        lib._closure_ready = True
    return lib


def _p(a: np.ndarray):
    assert a.dtype == REAL and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


def calcdef(arrays, *, ni, nj, nk, dx, dy, dz) -> None:
    """Writes arrays["defv"], arrays["defh"] in place."""
    rc = _lib().oracle_calcdef(ni, nj, nk, *(_p(arrays[n]) for n in DEFORMATION_INPUTS), dx, dy, dz,
                               _p(arrays["defv"]), _p(arrays["defh"]))
    if rc != 0:
        raise ValueError(f"oracle_calcdef failed ({rc})")


FLAT_DEFORMATION_INPUTS = ("u3d", "v3d", "w3d", "rho", "rf", "mf", "c1", "c2", "mh_profile")


def flat_calcdef(arrays, *, ni, nj, nk, dx, dy, rdz) -> None:
    """calcdef on a flat stretched column (enqueue_flat_calcdef,
    src/cm1core/cuda_gm1_flat_stretched_closure.py:524); writes defv, defh."""
    rc = _lib().oracle_flat_calcdef(ni, nj, nk, *(_p(arrays[n]) for n in FLAT_DEFORMATION_INPUTS), dx, dy, rdz,
                                    _p(arrays["defv"]), _p(arrays["defh"]))
    if rc != 0:
        raise ValueError(f"oracle_flat_calcdef failed ({rc})")


def moist_nm(arrays, *, ni, nj, nk, dz) -> dict[str, int]:
    """Writes nm, temperature, qt, thv, qvci and saturation_mask in place."""
    mask = arrays["saturation_mask"]
    assert mask.dtype == np.uint8 and mask.flags.c_contiguous
    counts = (ctypes.c_int64 * 4)()
    rc = _lib().oracle_moist_nm(ni, nj, nk, *(_p(arrays[n]) for n in NM_INPUTS), dz,
                                *(_p(arrays[n]) for n in NM_OUTPUTS), mask.ctypes.data, counts)
    if rc != 0:
        raise ValueError(f"oracle_moist_nm failed ({rc})")
    return {"saturated": counts[0], "liquid": counts[1], "mixed": counts[2], "ice": counts[3]}
