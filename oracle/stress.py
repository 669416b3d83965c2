"""ctypes driver of the SGS stress oracles (stress_oracle.c,
stress_terrain_oracle.c and the strain passes of closure_oracle.c) - TEST
INFRASTRUCTURE ONLY.  Restates enqueue_flat_calcdef's strain passes,
enqueue_flat_gettau and enqueue_flat_momentum_stress
(src/cm1core/cuda_gm1_flat_stretched_closure.py:76-114, :134-292, :524-618)
and, for the uniform column's terrain texts, the twins
cpu_sgs_stress_tendency_inplace (src/cm1core/cuda_sgs_stress_tendency.py:292)
and cpu_gm1_scalar_turbulence_inplace
(src/cm1core/cuda_gm1_scalar_turbulence.py:230)."""

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


SCALAR_TURBULENCE_INPUTS = ("th0", "tha", "qa", "rho", "rr", "rf", "mh", "mf", "khh", "khv")


def flat_scalar_turbulence(a, *, ni, nj, nk, numq, dx, dy, dz, dt) -> None:
    """turbs for theta and moisture rows 0..numq-1, added into thten1 and qten."""
    lib = load()
    if not getattr(lib, "_turbs_ready", False):
        i, f = ctypes.c_int, C_REAL
        lib.oracle_flat_scalar_turbulence.argtypes = [i, i, i, i] + [_F] * 10 + [f, f, f, f, _F, _F]
        lib.oracle_flat_scalar_turbulence.restype = i
        lib._turbs_ready = True
    for n in ("qa", "qten"):
        assert a[n].shape[0] >= numq and a[n].shape[1:] == (nk, nj, ni)
    rc = lib.oracle_flat_scalar_turbulence(ni, nj, nk, numq, *(_p(a[n]) for n in SCALAR_TURBULENCE_INPUTS), dx, dy,
                                           dz, dt, _p(a["thten1"]), _p(a["qten"]))
    if rc != 0:
        raise ValueError(f"oracle_flat_scalar_turbulence failed ({rc})")


# ------------------------------------------------------------------ Rayleigh
RAYLEIGH_INPUTS = ("tauh", "taus", "tauf", "u0", "v0", "ua", "va", "wa", "tha")


def rayleigh_coefficients(zh, zf, *, damping_start_m):
    """(tauh, taus, tauf): cpu_build_rayleigh_coefficients's formula
    (src/cm1core/cuda_rayleigh_held.py:264-383; CM1 param.F:8652-8671) in
    binary32 with numpy's float32 cosine; zf's last level is the top."""
    f = np.float32
    zh, zf = np.asarray(zh, f), np.asarray(zf, f)
    start, top = f(damping_start_m), zf[-1]

    def tau(z):
        ratio = np.divide(np.subtract(z, start, dtype=f), np.subtract(top[None], start, dtype=f), dtype=f)
        cosine = np.cos(np.multiply(f(np.pi), ratio, dtype=f), dtype=f)
        value = np.multiply(f(0.5), np.subtract(f(1.0), cosine, dtype=f), dtype=f)
        return np.where(z > start, value, f(0.0)).astype(f)

    th = tau(zh)
    return th, th.copy(), tau(zf)


def rayleigh_held(a, *, ni, nj, nk, rdalpha, profiles=False, add_momentum=False) -> None:
    """The irdamp = 1 held tendencies into uten1, vten1, wten1 and thten1."""
    lib = load()
    if not getattr(lib, "_rayleigh_ready", False):
        i, f = ctypes.c_int, C_REAL
        lib.oracle_rayleigh_held.argtypes = [i, i, i] + [_F] * 9 + [i, i, f] + [_F] * 4
        lib.oracle_rayleigh_held.restype = i
        lib._rayleigh_ready = True
    rc = lib.oracle_rayleigh_held(ni, nj, nk, *(_p(a[n]) for n in RAYLEIGH_INPUTS), 1 if profiles else 0,
                                  1 if add_momentum else 0, float(np.float32(rdalpha)),
                                  *(_p(a[n]) for n in ("uten1", "vten1", "wten1", "thten1")))
    if rc != 0:
        raise ValueError(f"oracle_rayleigh_held failed ({rc})")


def dissipative_heating(a, *, ni, nj, nk) -> None:
    """idiss = 1: the dissipative heating added into thten1."""
    lib = load()
    if not getattr(lib, "_diss_ready", False):
        i = ctypes.c_int
        lib.oracle_dissipative_heating.argtypes = [i, i, i] + [_F] * 5
        lib.oracle_dissipative_heating.restype = i
        lib._diss_ready = True
    rc = lib.oracle_dissipative_heating(ni, nj, nk, *(_p(a[n]) for n in ("dissten", "pi0", "ppi", "qa", "thten1")))
    if rc != 0:
        raise ValueError(f"oracle_dissipative_heating failed ({rc})")


# --------------------------------------------------- the terrain texts
TERRAIN_STRAIN_INPUTS = ("u3d", "v3d", "w3d", "rho", "rf", "gz", "rgz", "rgzu", "rgzv", "gx", "gy")
TERRAIN_MOMENTUM_INPUTS = TAU_NAMES + ("kmh", "kmv", "rho", "rf", "mh", "mf", "gz", "rgz", "gzu", "rgzu", "gzv",
                                       "rgzv", "gxu", "gyv", "u3d", "v3d", "w3d")
TERRAIN_TURBS_INPUTS = ("th0", "tha", "qa", "rho", "rr", "rf", "mh", "mf", "khh", "khv", "gz", "rgz", "rgzu",
                        "rgzv", "gx", "gxu", "gy", "gyv")


def _terrain_lib():
    lib = load()
    if not getattr(lib, "_terrain_stress_ready", False):
        i, f = ctypes.c_int, C_REAL
        lib.oracle_terrain_strain.argtypes = [i, i, i] + [_F] * 11 + [f, f, f] + [_F] * 6
        lib.oracle_terrain_strain.restype = i
        lib.oracle_terrain_gettau.argtypes = [i, i, i] + [_F] * 14
        lib.oracle_terrain_gettau.restype = i
        lib.oracle_terrain_momentum_stress.argtypes = [i, i, i] + [_F] * 23 + [f, f, f, f] + [_F] * 3
        lib.oracle_terrain_momentum_stress.restype = i
        lib.oracle_terrain_scalar_turbulence.argtypes = [i, i, i, i] + [_F] * 18 + [f, f, f, f, _F, _F]
        lib.oracle_terrain_scalar_turbulence.restype = i
        lib._terrain_stress_ready = True
    return lib


def terrain_strain(a, *, ni, nj, nk, dx, dy, dz) -> None:
    rc = _terrain_lib().oracle_terrain_strain(ni, nj, nk, *(_p(a[n]) for n in TERRAIN_STRAIN_INPUTS), dx, dy, dz,
                                              *(_p(a[n]) for n in STRAIN_NAMES))
    if rc != 0:
        raise ValueError(f"oracle_terrain_strain failed ({rc})")


def terrain_gettau(a, *, ni, nj, nk) -> None:
    rc = _terrain_lib().oracle_terrain_gettau(ni, nj, nk, *(_p(a[n]) for n in STRAIN_NAMES), _p(a["kmh"]),
                                              _p(a["kmv"]), *(_p(a[n]) for n in TAU_NAMES))
    if rc != 0:
        raise ValueError(f"oracle_terrain_gettau failed ({rc})")


def terrain_momentum_stress(a, *, ni, nj, nk, dx, dy, dz, dt) -> None:
    rc = _terrain_lib().oracle_terrain_momentum_stress(ni, nj, nk, *(_p(a[n]) for n in TERRAIN_MOMENTUM_INPUTS), dx, dy,
                                                       dz, dt, *(_p(a[n]) for n in TENDENCY_NAMES))
    if rc != 0:
        raise ValueError(f"oracle_terrain_momentum_stress failed ({rc})")


def terrain_sgs_stress(a, *, ni, nj, nk, dx, dy, dz, dt) -> None:
    terrain_strain(a, ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, dz=dz)
    terrain_gettau(a, ni=ni, nj=nj, nk=nk)
    terrain_momentum_stress(a, ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, dz=dz, dt=dt)


def terrain_scalar_turbulence(a, *, ni, nj, nk, numq, dx, dy, dz, dt) -> None:
    rc = _terrain_lib().oracle_terrain_scalar_turbulence(ni, nj, nk, numq, *(_p(a[n]) for n in TERRAIN_TURBS_INPUTS),
                                                         dx, dy, dz, dt, _p(a["thten1"]), _p(a["qten"]))
    if rc != 0:
        raise ValueError(f"oracle_terrain_scalar_turbulence failed ({rc})")
