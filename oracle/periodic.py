"""ctypes driver of liboracle_gm1.so, the C restatement of the reference's
NumPy twins for the serial-periodic dry lane - TEST INFRASTRUCTURE ONLY.

Mirrors the reference CPU entry points:
  cpu_sound3_periodic_three_stage_inplace (src/cm1core/cuda_sound3_periodic.py:1071)
  cpu_psolver3_trajectory_inplace         (src/cm1core/cuda_psolver3_trajectory.py:761)
on dictionaries of float32 numpy arrays with the reference names and shapes.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# Working precision of the oracle build this process loads: binary32, the
# reference twins' arithmetic (liboracle_gm1.so), or, with
# GM1B_ORACLE_REAL=f64, the same operators evaluated in binary64
# (liboracle_gm1_f64.so, the FP64 run the float32 fields are measured against).
F64 = os.environ.get("GM1B_ORACLE_REAL", "f32") == "f64"
REAL = np.float64 if F64 else np.float32
C_REAL = ctypes.c_double if F64 else ctypes.c_float
LIB_PATH = HERE / ("liboracle_gm1_f64.so" if F64 else "liboracle_gm1.so")

# Field order of gm1b_periodic_arrays (include/gm1b.h): the reference's
# ALL_ARRAY_NAMES order.
NAMES = (
    "mh", "rr0", "rf0", "c1", "c2", "mf", "piadv", "ppterm", "thv", "ppten",
    "ppi", "pp3d", "ppx", "ppd", "qk", "pk1", "pk2", "mm", "fpk", "divh",
    "hadvp", "elim_c", "elim_d", "tri_aa", "tri_bb", "tri_cc", "tri_dd",
    "tri_pivot", "tri_residual",
    "wten", "wa", "w3d", "rrw",
    "ua", "u3d", "uten", "rru",
    "va", "v3d", "vten", "rrv",
    "dtu0", "dtv0", "uf", "vf", "uh", "vh",
    "pi0", "rho0", "rrf0", "th0", "rth0", "tha", "th3d", "sadv", "thten", "divx",
)

CP = 1005.7
ALPH = 0.60
KDIV = 0.10
SMEPS = 1.0e-30


class PeriodicArrays(ctypes.Structure):
    _fields_ = [(name, ctypes.POINTER(C_REAL)) for name in NAMES]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        lib = ctypes.CDLL(str(LIB_PATH))
        f = C_REAL
        i = ctypes.c_int
        p = ctypes.POINTER(PeriodicArrays)
        lib.oracle_stage_schedule.argtypes = [f, i, i, ctypes.POINTER(i), ctypes.POINTER(f)]
        lib.oracle_stage_schedule.restype = i
        lib.oracle_rk_stage_dt.argtypes = [f, i]
        lib.oracle_rk_stage_dt.restype = f
        lib.oracle_sound3_periodic_stage.argtypes = [p, i, i, i, f, i, i, f, f, f, f, f, f, f]
        lib.oracle_sound3_periodic_stage.restype = i
        lib.oracle_traj_stage.argtypes = [p, i, i, i, f, i, i, f, f, f, ctypes.c_uint]
        lib.oracle_traj_stage.restype = i
        lib.oracle_traj_post_step.argtypes = [p, i, i, i, i, i]
        lib.oracle_traj_post_step.restype = None
        lib.oracle_traj_steps.argtypes = [p, i, i, i, i, f, i, f, f, f, ctypes.c_uint]
        lib.oracle_traj_steps.restype = i
        lib.oracle_set_threads.argtypes = [i]
        lib.oracle_set_threads.restype = None
        lib.oracle_max_threads.argtypes = []
        lib.oracle_max_threads.restype = i
        _lib = lib
    return _lib


def set_threads(n: int) -> None:
    load().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(load().oracle_max_threads())


def _struct(arrays: dict[str, np.ndarray], names=NAMES) -> PeriodicArrays:
    s = PeriodicArrays()
    for name in names:
        a = arrays.get(name)
        if a is None:
            continue
        if a.dtype != REAL or not a.flags.c_contiguous or not a.flags.writeable:
            raise ValueError(f"{name} must be a writable C-contiguous float32 array")
        setattr(s, name, a.ctypes.data_as(ctypes.POINTER(C_REAL)))
    return s


def stage_schedule(dt: float, nsound: int, nrk: int) -> tuple[int, float]:
    n = ctypes.c_int()
    d = C_REAL()
    if load().oracle_stage_schedule(dt, nsound, nrk, ctypes.byref(n), ctypes.byref(d)) != 0:
        raise ValueError("invalid acoustic schedule arguments")
    return n.value, float(d.value)


def rk_stage_dt(dt: float, nrk: int) -> float:
    return float(load().oracle_rk_stage_dt(dt, nrk))


def sound3_periodic_stage(arrays, *, ni, nj, nk, dt, nsound, nrk, rdx, rdy, rdz,
                          cp=CP, alph=ALPH, kdiv=KDIV, smeps=SMEPS) -> int:
    s = _struct(arrays, NAMES[:47])
    n = load().oracle_sound3_periodic_stage(ctypes.byref(s), ni, nj, nk, dt, nsound, nrk,
                                            rdx, rdy, rdz, cp, alph, kdiv, smeps)
    if n < 0:
        raise ValueError("invalid acoustic schedule arguments")
    return n


def sound3_periodic_three_stage(arrays, **kwargs) -> list[int]:
    return [sound3_periodic_stage(arrays, nrk=nrk, **kwargs) for nrk in (1, 2, 3)]


def traj_stage(arrays, *, ni, nj, nk, dt, nsound, nrk, dx, dy, dz, ablations=0) -> int:
    s = _struct(arrays)
    n = load().oracle_traj_stage(ctypes.byref(s), ni, nj, nk, dt, nsound, nrk, dx, dy, dz, ablations)
    if n < 0:
        raise ValueError("invalid trajectory arguments")
    return n


def traj_post_step(arrays, *, ni, nj, nk, ablations=0) -> None:
    s = _struct(arrays)
    load().oracle_traj_post_step(ctypes.byref(s), ni, nj, nk, int(not (ablations & 16)),
                                 int(not (ablations & 32)))


def traj_steps(arrays, *, ni, nj, nk, steps, dt, nsound, dx, dy, dz, ablations=0) -> None:
    s = _struct(arrays)
    if load().oracle_traj_steps(ctypes.byref(s), ni, nj, nk, steps, dt, nsound, dx, dy, dz, ablations) != 0:
        raise ValueError("invalid trajectory arguments")
