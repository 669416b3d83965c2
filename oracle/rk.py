"""ctypes driver of the scalar/moisture RK oracle (rk_oracle.c) - TEST
INFRASTRUCTURE ONLY.  Mirrors cpu_theta_transport_scalar_inplace,
cpu_compose_scalar_moist_rk_stage_inplace and cpu_pdef_direction_inplace
(src/cm1core/cuda_scalar_moist_rk.py:255,283,352)."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)
AXES = {"x": 0, "y": 1, "z": 2}


def _p(a):
    assert a.dtype == REAL and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


def _lib():
    lib = load()
    if not getattr(lib, "_rk_ready", False):
        i, f = ctypes.c_int, C_REAL
        lib.oracle_theta_pack.argtypes = [_F, _F, _F, i, i, i]
        lib.oracle_theta_pack.restype = None
        lib.oracle_rk_compose.argtypes = [_F] * 9 + [ctypes.c_size_t, i, f]
        lib.oracle_rk_compose.restype = None
        lib.oracle_pdef_direction.argtypes = [_F] * 8 + [i, i, i, i, f, f]
        lib.oracle_pdef_direction.restype = None
        lib._rk_ready = True
    return lib


def theta_pack(th0, th3d, padded, *, ni, nj, nk):
    _lib().oracle_theta_pack(_p(th0), _p(th3d), _p(padded), ni, nj, nk)


def rk_stage_dt(dt, nrk):
    return float(np.float32(np.float32(dt) / np.float32(4 - nrk)))


def compose(theta_a, q_a, theta_held, q_held, theta_divterm, theta_adv, q_adv, theta_cur, q_cur, *, nrk, dt):
    nq = q_a.shape[0]
    _lib().oracle_rk_compose(_p(theta_a), _p(theta_held), _p(theta_divterm), _p(theta_adv), _p(theta_cur), _p(q_a),
                             _p(q_held), _p(q_adv), _p(q_cur), theta_a.size, nq, rk_stage_dt(dt, nrk))


def pdef_direction(scalar_a, scalar_padded, rho0, gz, rgz, mass_flux, directional, candidate, *, axis, dt, spacing):
    nk, nj, ni = scalar_a.shape
    _lib().oracle_pdef_direction(_p(scalar_a), _p(scalar_padded), _p(rho0), _p(gz), _p(rgz), _p(mass_flux),
                                 _p(directional), _p(candidate), ni, nj, nk, AXES[axis], dt, spacing)
