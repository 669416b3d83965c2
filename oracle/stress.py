"""ctypes driver of the flat-column SGS stress oracle (stress_oracle.c and
the strain passes of closure_oracle.c) - TEST INFRASTRUCTURE ONLY.
Restates enqueue_flat_calcdef's strain passes, enqueue_flat_gettau and
enqueue_flat_momentum_stress (src/cm1core/cuda_gm1_flat_stretched_closure.py:
76-114, :134-292, :524-618)."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)

STRAIN_INPUTS = ("u3d", "v3d", "w3d", "rho", "rf", "mf", "mh_profile")
STRAIN_NAMES = ("s11", "s22", "s33", "s12", "s13", "s23")
TAU_NAMES = ("t11", "t22", "t33", "t12", "t13", "t23")
MOMENTUM_INPUTS = TAU_NAMES + ("kmh", "kmv", "rho", "rf", "mh", "mf", "u3d", "v3d", "w3d")
TENDENCY_NAMES = ("uten", "vten", "wten")


def stress_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    cell, face = (nk, nj, ni), (nk + 1, nj, ni)
    return {"u3d": (nk, nj, ni + 1), "v3d": (nk, nj + 1, ni), "w3d": face, "rho": cell, "rf": face, "mh": cell,
            "mf": face, "mh_profile": (nk + 2,), "kmh": face, "kmv": face,
            **{n: cell for n in ("s11", "s22", "s33", "t11", "t22", "t33")},
            "s12": (nk, nj + 1, ni + 1), "t12": (nk, nj + 1, ni + 1), "s13": (nk + 1, nj, ni + 1),
            "t13": (nk + 1, nj, ni + 1), "s23": (nk + 1, nj + 1, ni), "t23": (nk + 1, nj + 1, ni),
            "uten": (nk, nj, ni + 1), "vten": (nk, nj + 1, ni), "wten": face}


def _lib():
    lib = load()
    if not getattr(lib, "_stress_ready", False):
        i, f = ctypes.c_int, C_REAL
        lib.oracle_flat_strain.argtypes = [i, i, i] + [_F] * 7 + [f, f, f] + [_F] * 6
        lib.oracle_flat_strain.restype = i
        lib.oracle_flat_gettau.argtypes = [i, i, i] + [_F] * 14
        lib.oracle_flat_gettau.restype = i
        lib.oracle_flat_momentum_stress.argtypes = [i, i, i] + [_F] * 15 + [f, f, f, f] + [_F] * 3
        lib.oracle_flat_momentum_stress.restype = i
        lib._stress_ready = True
    return lib


def _p(a: np.ndarray):
    assert a.dtype == REAL and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


def flat_strain(a, *, ni, nj, nk, dx, dy, rdz) -> None:
    """The strain carriers s11..s23 (face levels 0 and nk of s13/s23 are
    left as they are)."""
    rc = _lib().oracle_flat_strain(ni, nj, nk, *(_p(a[n]) for n in STRAIN_INPUTS), dx, dy, rdz,
                                   *(_p(a[n]) for n in STRAIN_NAMES))
    if rc != 0:
        raise ValueError(f"oracle_flat_strain failed ({rc})")


def flat_gettau(a, *, ni, nj, nk) -> None:
    """t11..t23 from s11..s23, kmh and kmv."""
    rc = _lib().oracle_flat_gettau(ni, nj, nk, *(_p(a[n]) for n in STRAIN_NAMES), _p(a["kmh"]), _p(a["kmv"]),
                                   *(_p(a[n]) for n in TAU_NAMES))
    if rc != 0:
        raise ValueError(f"oracle_flat_gettau failed ({rc})")


def flat_momentum_stress(a, *, ni, nj, nk, dx, dy, rdz, dt) -> None:
    """turbu, turbv and turbw added into uten, vten and wten."""
    rc = _lib().oracle_flat_momentum_stress(ni, nj, nk, *(_p(a[n]) for n in MOMENTUM_INPUTS), dx, dy, rdz, dt,
                                            *(_p(a[n]) for n in TENDENCY_NAMES))
    if rc != 0:
        raise ValueError(f"oracle_flat_momentum_stress failed ({rc})")


def flat_sgs_stress(a, *, ni, nj, nk, dx, dy, rdz, dt) -> None:
    """strain, gettau and the momentum stress in that order."""
    flat_strain(a, ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, rdz=rdz)
    flat_gettau(a, ni=ni, nj=nj, nk=nk)
    flat_momentum_stress(a, ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, rdz=rdz, dt=dt)


def zeros(ni, nj, nk, names) -> dict[str, np.ndarray]:
    sh = stress_shapes(ni, nj, nk)
    return {n: np.zeros(sh[n], REAL) for n in names}
