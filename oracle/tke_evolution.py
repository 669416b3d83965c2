"""ctypes driver of the TKE-evolution oracle (tke_evolution_oracle.c) - TEST
INFRASTRUCTURE ONLY.  Mirrors cpu_tke_evolution_inplace
(src/cm1core/cuda_tke_evolution.py:206): turbt into tketen, then three RK
stages from tke3d towards tkea, then the commit tke3d = tkea = result."""

from __future__ import annotations

import ctypes
import hashlib

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)
DIFFUSION_NAMES = ("tke3d", "kmh", "kmv", "rho", "rf", "mh", "mf", "gz", "rgz", "rgzu", "rgzv", "tketen")
STAGE_NAMES = ("tkea", "tketen", "c1", "c2", "rrf0", "gz", "rru", "rrv", "rrw", "divx")


def _lib():
    lib = load()
    if not getattr(lib, "_tkeevo_ready", False):
        i, f = ctypes.c_int, C_REAL
        lib.oracle_tke_diffusion.argtypes = [i, i, i] + [_F] * 12 + [f, f, f, f]
        lib.oracle_tke_diffusion.restype = i
        lib.oracle_tke_rk_stage.argtypes = [i, i, i] + [_F] * 12 + [i, f, f, f, f]
        lib.oracle_tke_rk_stage.restype = i
        lib.oracle_tke_diffusion_flat.argtypes = [i, i, i] + [_F] * 8 + [f, f, f, f]
        lib.oracle_tke_diffusion_flat.restype = i
        lib.oracle_tke_rk_stage_flat.argtypes = [i, i, i] + [_F] * 11 + [i, f, f, f, f]
        lib.oracle_tke_rk_stage_flat.restype = i
        lib._tkeevo_ready = True
    return lib


def _p(a):
    assert a.dtype == REAL and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


def tke_diffusion(a, *, ni, nj, nk, dx, dy, dz, dt) -> None:
    rc = _lib().oracle_tke_diffusion(ni, nj, nk, *(_p(a[n]) for n in DIFFUSION_NAMES), dx, dy, dz, dt)
    if rc != 0:
        raise ValueError(f"oracle_tke_diffusion failed ({rc})")


def tke_rk_stage(a, cur, nxt, *, ni, nj, nk, nrk, dx, dy, dz, dt) -> None:
    rc = _lib().oracle_tke_rk_stage(ni, nj, nk, _p(cur), *(_p(a[n]) for n in STAGE_NAMES), _p(nxt), nrk,
                                    dx, dy, dz, dt)
    if rc != 0:
        raise ValueError(f"oracle_tke_rk_stage failed ({rc})")


def tke_evolution(a, *, ni, nj, nk, dx, dy, dz, dt) -> list[str]:
    """The whole operator in place; returns the SHA-256 of each stage result."""
    tke_diffusion(a, ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, dz=dz, dt=dt)
    cur = a["tke3d"].copy()
    hashes = []
    for nrk in (1, 2, 3):
        nxt = np.zeros_like(cur)
        tke_rk_stage(a, cur, nxt, ni=ni, nj=nj, nk=nk, nrk=nrk, dx=dx, dy=dy, dz=dz, dt=dt)
        cur = nxt
        hashes.append(hashlib.sha256(cur.astype("<f4", copy=False).tobytes()).hexdigest())
    a["tke3d"][...] = cur
    a["tkea"][...] = cur
    return hashes


FLAT_DIFFUSION_NAMES = ("tke3d", "kmh", "kmv", "rho", "rf", "mh", "mf", "tketen")
FLAT_STAGE_NAMES = ("tkea", "tketen", "c2", "rrf0", "rru", "rrv", "rrw", "divx")


def tke_diffusion_flat(a, *, ni, nj, nk, dx, dy, rdz, dt) -> None:
    """turbt on a flat stretched column (gm1_flat_turbt_v1,
    src/cm1core/cuda_gm1_flat_stretched_closure.py:314); adds into tketen."""
    rc = _lib().oracle_tke_diffusion_flat(ni, nj, nk, *(_p(a[n]) for n in FLAT_DIFFUSION_NAMES), dx, dy, rdz, dt)
    if rc != 0:
        raise ValueError(f"oracle_tke_diffusion_flat failed ({rc})")


def tke_rk_stage_flat(a, mf_profile, cur, nxt, *, ni, nj, nk, nrk, dx, dy, rdz, dt) -> None:
    """One RK stage on a flat stretched column (gm1_flat_tke_advw_rk_v1)."""
    rc = _lib().oracle_tke_rk_stage_flat(ni, nj, nk, _p(cur), *(_p(a[n]) for n in FLAT_STAGE_NAMES),
                                         _p(mf_profile), _p(nxt), nrk, dx, dy, rdz, dt)
    if rc != 0:
        raise ValueError(f"oracle_tke_rk_stage_flat failed ({rc})")
