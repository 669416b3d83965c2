"""ctypes driver of the moist-step pieces of the oracle
(moist_step_oracle.c, terrain_open_oracle.c's fills) - TEST INFRASTRUCTURE
ONLY."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)
POST_NAMES = ("rru", "rrv", "rrw", "rgzu", "rgzv", "dzdx", "dzdy", "gz", "rho0_3d", "rf0", "thterm", "divergence",
              "theta_divergence_term", "divx")
CHAIN_NAMES = ("scalar_a", "scalar_padded", "rho0_3d", "gz", "rgz", "rr0", "c1", "c2", "divx", "rru", "rrv", "rrw",
               "fx", "fy", "fz", "advx", "advy", "advz", "candidate", "advection")
HELD_NAMES = ("th0", "pi0", "rho", "ppi", "tha", "qa", "qpten", "qtten", "qvten", "qcten", "thheld", "qheld", "ppten")
FILL = {"pressure": 0, "scalar": 1, "u": 2, "v": 3, "w": 4, "w_keep_ends": 5}


def _struct(names):
    class S(ctypes.Structure):
        _fields_ = [(n, _F) for n in names]
    return S


_Post, _Chain, _Held = _struct(POST_NAMES), _struct(CHAIN_NAMES), _struct(HELD_NAMES)


def _p(a):
    assert a.dtype == REAL and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


def _lib():
    lib = load()
    if not getattr(lib, "_ms_ready", False):
        c = ctypes
        lib.oracle_open_fill.argtypes = [c.c_int] * 4 + [_F]
        lib.oracle_moist_buoyancy.argtypes = [c.c_int] * 3 + [_F] * 8
        lib.oracle_post_acoustic_flux.argtypes = [c.c_int] * 3 + [c.POINTER(_Post)] + [C_REAL] * 3
        lib.oracle_pdef_moisture_chain.argtypes = [c.c_int] * 3 + [c.POINTER(_Chain)] + [C_REAL] * 4 + \
            [c.c_double, c.c_uint, c.c_int]
        lib.oracle_pdef_moisture_directional.argtypes = lib.oracle_pdef_moisture_chain.argtypes
        lib.oracle_pdef_moisture_directional.restype = None
        lib.oracle_pdef_moisture_chain_column.argtypes = [c.c_int] * 3 + [c.POINTER(_Chain)] + [C_REAL] * 3 + \
            [c.c_double, c.c_uint, c.c_int, c.c_int, _F, _F, C_REAL]
        lib.oracle_pdef_moisture_chain_column.restype = None
        lib.oracle_post_acoustic_flux_column.argtypes = [c.c_int] * 3 + [c.POINTER(_Post)] + [C_REAL] * 2 + \
            [c.c_int] + [_F] * 5 + [C_REAL, _F, C_REAL]
        lib.oracle_post_acoustic_flux_column.restype = None
        lib.oracle_moist_buoyancy_flat.argtypes = [c.c_int] * 3 + [_F] * 4
        lib.oracle_moist_buoyancy_flat.restype = None
        lib.oracle_held_compose.argtypes = [c.c_int] * 3 + [c.POINTER(_Held), C_REAL]
        lib.oracle_solve3_density.argtypes = [c.c_int] * 3 + [_F] * 5
        lib.oracle_pack_scalar.argtypes = [c.c_int] * 3 + [_F] * 2
        lib.oracle_bcwsfc.argtypes = [c.c_int] * 3 + [_F] * 6
        lib.oracle_w_level1_fill.argtypes = [c.c_int] * 3 + [_F]
        for f in ("oracle_bcwsfc", "oracle_w_level1_fill", "oracle_open_fill", "oracle_moist_buoyancy", "oracle_post_acoustic_flux",
                  "oracle_pdef_moisture_chain", "oracle_held_compose", "oracle_solve3_density", "oracle_pack_scalar"):
            getattr(lib, f).restype = None
        lib._ms_ready = True
    return lib


def open_fill(q, kind, *, ni, nj, nk):
    _lib().oracle_open_fill(ni, nj, nk, FILL[kind], _p(q))


def moist_buoyancy(dum8, c1, c2, gxu, gyv, uten, vten, wten, *, ni, nj, nk):
    _lib().oracle_moist_buoyancy(ni, nj, nk, *(_p(x) for x in (dum8, c1, c2, gxu, gyv, uten, vten, wten)))


def post_acoustic_flux(a, *, ni, nj, nk, dx, dy, dz):
    s = _Post(**{n: _p(a[n]) for n in POST_NAMES})
    _lib().oracle_post_acoustic_flux(ni, nj, nk, ctypes.byref(s), dx, dy, dz)


def post_acoustic_flux_column(a, column, *, ni, nj, nk, dx, dy):
    """getdiv/getdivx on a stretched column: ``column`` holds flat, rho0p and
    sigma/sigmaf/rds/rdsf/ztop (terrain branch) or mh/rdz (flat column)."""
    s = _Post(**{n: _p(a[n]) for n in POST_NAMES})
    keep = {n: np.ascontiguousarray(column[n], dtype=REAL) for n in ("rho0p", "sigma", "sigmaf", "rds", "rdsf",
                                                                           "mh") if column.get(n) is not None}
    ptr = {n: (_p(keep[n]) if n in keep else None) for n in ("rho0p", "sigma", "sigmaf", "rds", "rdsf", "mh")}
    _lib().oracle_post_acoustic_flux_column(ni, nj, nk, ctypes.byref(s), dx, dy, 1 if column["flat"] else 0,
                                            ptr["rho0p"], ptr["sigma"], ptr["sigmaf"], ptr["rds"], ptr["rdsf"],
                                            float(column.get("ztop", 0.0)), ptr["mh"], float(column.get("rdz", 0.0)))


def moist_buoyancy_flat(dum8, c1, c2, wten, *, ni, nj, nk):
    _lib().oracle_moist_buoyancy_flat(ni, nj, nk, _p(dum8), _p(c1), _p(c2), _p(wten))


def pdef_moisture_chain(a, *, ni, nj, nk, dttmp, dx, dy, dz, weps, lateral_obc, pdefweno):
    s = _Chain(**{n: _p(a[n]) for n in CHAIN_NAMES})
    _lib().oracle_pdef_moisture_chain(ni, nj, nk, ctypes.byref(s), dttmp, dx, dy, dz, weps, lateral_obc, pdefweno)


def pdef_moisture_chain_column(a, *, ni, nj, nk, dttmp, dx, dy, weps, lateral_obc, pdefweno, flat, profile, rdz=0.0):
    """The chain on a stretched column: flat=False takes profile = rdsf
    (nk+3 words, CM1 indexing), flat=True profile = mh (nk+2 words) and rdz."""
    s = _Chain(**{n: _p(a[n]) for n in CHAIN_NAMES})
    prof = np.ascontiguousarray(profile, dtype=REAL)
    _lib().oracle_pdef_moisture_chain_column(ni, nj, nk, ctypes.byref(s), dttmp, dx, dy, weps, lateral_obc, pdefweno,
                                             2 if flat else 1, None if flat else _p(prof), _p(prof) if flat else None,
                                             rdz)


def pdef_moisture_directional(a, *, ni, nj, nk, dttmp, dx, dy, dz, weps, lateral_obc, pdefweno):
    """The chain up to the directional advection (advx/advy/advz before any repair)."""
    s = _Chain(**{n: _p(a[n]) for n in CHAIN_NAMES})
    _lib().oracle_pdef_moisture_directional(ni, nj, nk, ctypes.byref(s), dttmp, dx, dy, dz, weps, lateral_obc, pdefweno)


def held_compose(a, *, ni, nj, nk, dt):
    s = _Held(**{n: _p(a[n]) for n in HELD_NAMES})
    _lib().oracle_held_compose(ni, nj, nk, ctypes.byref(s), dt)


def solve3_density(rho, c1, c2, rr, rf, *, ni, nj, nk):
    _lib().oracle_solve3_density(ni, nj, nk, *(_p(x) for x in (rho, c1, c2, rr, rf)))


def pack_scalar(s, padded, *, ni, nj, nk):
    _lib().oracle_pack_scalar(ni, nj, nk, _p(s), _p(padded))


def bcwsfc(u3d, v3d, w3d, gz, dzdx, dzdy, *, ni, nj, nk):
    _lib().oracle_bcwsfc(ni, nj, nk, *(_p(x) for x in (u3d, v3d, w3d, gz, dzdx, dzdy)))


def w_level1_fill(w3d, *, ni, nj, nk):
    _lib().oracle_w_level1_fill(ni, nj, nk, _p(w3d))
