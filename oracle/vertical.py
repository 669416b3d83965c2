"""ctypes driver of the vertical-coordinate oracle (oracle/vertical_oracle.c)
- TEST INFRASTRUCTURE ONLY.

Mirrors build_vertical_levels (src/cm1core/cm1_vertical_grid.py:780) for
stretch_z 0 and 1 and derive_stretch_z1 (src/cm1core/cuda_stretch_z1.py:130)
on float32 numpy arrays with CM1's indexing: zf, sigmaf, mf, rmf, rdsf hold
nk+3 words, zh, sigma, mh, rmh, rds nk+2.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .periodic import load

PROFILES = ("zf", "zh", "sigmaf", "sigma", "mh", "mf", "rmh", "rmf", "rds", "rdsf")
LONG = ("zf", "sigmaf", "mf", "rmf", "rdsf")


class Derived(ctypes.Structure):
    _fields_ = [("nk1", ctypes.c_int32), ("nk2", ctypes.c_int32), ("nk3", ctypes.c_int32),
                ("nominal", ctypes.c_float), ("c1", ctypes.c_float), ("c2", ctypes.c_float)]


def _bind():
    lib = load()
    if not getattr(lib, "_vertical_bound", False):
        f, i = ctypes.c_float, ctypes.c_int
        fp = ctypes.POINTER(ctypes.c_float)
        lib.oracle_derive_stretch_z1.argtypes = [i] + [f] * 6 + [ctypes.POINTER(Derived)]
        lib.oracle_derive_stretch_z1.restype = i
        lib.oracle_vertical_levels.argtypes = [i, i] + [f] * 6 + [fp] * 12
        lib.oracle_vertical_levels.restype = i
        lib._vertical_bound = True
    return lib


def derive_stretch_z1(nk, dz, ztop, str_bot, str_top, dz_bot, dz_top) -> tuple[int, Derived]:
    d = Derived()
    rc = _bind().oracle_derive_stretch_z1(nk, dz, ztop, str_bot, str_top, dz_bot, dz_top, ctypes.byref(d))
    return rc, d


def vertical_levels(stretch_z, nk, dz, ztop, str_bot=0.0, str_top=0.0, dz_bot=0.0,
                    dz_top=0.0) -> tuple[int, dict[str, np.ndarray]]:
    out = {n: np.zeros(nk + 3 if n in LONG else nk + 2, np.float32) for n in PROFILES}
    out["cgs"] = np.zeros(3, np.float32)
    out["cgt"] = np.zeros(3, np.float32)
    ptr = [out[n].ctypes.data_as(ctypes.POINTER(ctypes.c_float)) for n in PROFILES + ("cgs", "cgt")]
    rc = _bind().oracle_vertical_levels(stretch_z, nk, dz, ztop, str_bot, str_top, dz_bot, dz_top, *ptr)
    return rc, out
