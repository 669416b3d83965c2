"""ctypes driver of the analytic initial-state oracle (init_oracle.c) - TEST
INFRASTRUCTURE ONLY.  Mirrors weisman_klemp_column_with_iterations,
analytic_shear_u/v and build_theta_perturbation iinit=1
(rust/cm1-state/src/storm_initialization.rs:194,354,373;
rust/cm1-state/src/initial_perturbation.rs:449-466)."""

from __future__ import annotations

import ctypes

import numpy as np

from oracle.periodic import load

_F = ctypes.POINTER(ctypes.c_float)
COLUMN_NAMES = ("th0", "qv0", "thv0", "pi0", "prs0", "t0", "rh0")


def _lib():
    lib = load()
    if not getattr(lib, "_init_ready", False):
        i, f = ctypes.c_int, ctypes.c_float
        lib.oracle_wk_column.argtypes = [i, _F, i, i] + [_F] * 7
        lib.oracle_wk_column.restype = i
        lib.oracle_wk_surface.argtypes = [_F]
        lib.oracle_wk_surface.restype = None
        lib.oracle_analytic_shear.argtypes = [i, _F, _F, _F, _F]
        lib.oracle_analytic_shear.restype = None
        lib.oracle_theta_bubble.argtypes = [i, i, i, _F, _F, _F, f, f, f, f, f, f, _F]
        lib.oracle_theta_bubble.restype = None
        lib._init_ready = True
    return lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_F)


def wk_column(heights, imoist: int = 1, iterations: int = 20) -> dict[str, np.ndarray]:
    z = np.ascontiguousarray(heights, dtype=np.float32)
    out = {n: np.zeros(z.size, np.float32) for n in COLUMN_NAMES}
    rc = _lib().oracle_wk_column(z.size, _p(z), imoist, iterations, *(_p(out[n]) for n in COLUMN_NAMES))
    if rc != 0:
        raise ValueError("oracle_wk_column refused its arguments")
    return out


def wk_surface() -> np.ndarray:
    out = np.zeros(3, np.float32)
    _lib().oracle_wk_surface(_p(out))
    return out


def analytic_shear(zu, zv) -> tuple[np.ndarray, np.ndarray]:
    zu = np.ascontiguousarray(zu, dtype=np.float32)
    zv = np.ascontiguousarray(zv, dtype=np.float32)
    assert zu.size == zv.size
    u = np.zeros(zu.size, np.float32)
    v = np.zeros(zv.size, np.float32)
    _lib().oracle_analytic_shear(zu.size, _p(zu), _p(zv), _p(u), _p(v))
    return u, v


def theta_bubble(xh, yh, zh, *, xc, yc, zc, hrad, zrad, amp) -> np.ndarray:
    xh = np.ascontiguousarray(xh, dtype=np.float32)
    yh = np.ascontiguousarray(yh, dtype=np.float32)
    zh = np.ascontiguousarray(zh, dtype=np.float32)
    tha = np.zeros((zh.size, yh.size, xh.size), np.float32)
    _lib().oracle_theta_bubble(xh.size, yh.size, zh.size, _p(xh), _p(yh), _p(zh), xc, yc, zc, hrad, zrad, amp,
                               _p(tha))
    return tha
