"""Loader of libgm1b.so, the CUDA library behind every operator here.

There is no fallback: if the library is missing or was built for another ABI,
every operator raises.  Build it with ``python -m gm1_b200.csrc.build``.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

from .arrays import ALL_ARRAY_NAMES

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libgm1b.so"
ABI_VERSION = 1

GM1B_OK = 0
GM1B_ERR_ARGUMENT = -1
GM1B_FLAG_SCRATCH_OUTPUTS = 1
GM1B_FLAG_MULTI_LAUNCH_STAGE = 2

# ablation bits of include/gm1b.h, keyed by the reference field names
ABLATION_BITS = {
    "momentum_advection": 1,
    "scalar_advection": 2,
    "base_theta_advection": 4,
    "buoyancy": 8,
    "post_step_ppx": 16,
    "carrier_promotion": 32,
}


class KernelStat(ctypes.Structure):
    """gm1b_kernel_stat of the launch profiler."""

    _fields_ = [("name", ctypes.c_char * 48), ("launches", ctypes.c_int32), ("total_ms", ctypes.c_double)]


class PeriodicArrays(ctypes.Structure):
    """gm1b_periodic_arrays: one device pointer per reference array name."""

    _fields_ = [(name, ctypes.c_void_p) for name in ALL_ARRAY_NAMES]


_lib: ctypes.CDLL | None = None


class Gm1bError(RuntimeError):
    """A libgm1b.so entry point returned a non-zero status."""


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: the CUDA library must be built "
            "(python -m gm1_b200.csrc.build); there is no CPU fallback"
        )
    handle = ctypes.CDLL(str(LIB_PATH))
    i32, u32, f32, vp = ctypes.c_int32, ctypes.c_uint32, ctypes.c_float, ctypes.c_void_p
    pa = ctypes.POINTER(PeriodicArrays)
    handle.gm1b_abi_version.argtypes = []
    handle.gm1b_abi_version.restype = i32
    handle.gm1b_last_error.argtypes = []
    handle.gm1b_last_error.restype = ctypes.c_char_p
    handle.gm1b_sound3_stage_schedule.argtypes = [f32, i32, i32, ctypes.POINTER(i32), ctypes.POINTER(f32)]
    handle.gm1b_sound3_stage_schedule.restype = i32
    handle.gm1b_rk_stage_dt.argtypes = [f32, i32]
    handle.gm1b_rk_stage_dt.restype = f32
    handle.gm1b_sound3_periodic_three_stage.argtypes = [
        i32, i32, i32, pa, f32, i32, f32, f32, f32, f32, f32, f32, u32, vp,
    ]
    handle.gm1b_sound3_periodic_three_stage.restype = i32
    handle.gm1b_psolver3_trajectory.argtypes = [
        i32, i32, i32, pa, i32, f32, i32, f32, f32, f32, u32, u32, vp,
    ]
    handle.gm1b_psolver3_trajectory.restype = i32
    handle.gm1b_sound3_periodic_three_stage_checked.argtypes = [
        i32, i32, i32, pa, f32, i32, f32, f32, f32, f32, f32, f32, u32, i32, vp, vp,
    ]
    handle.gm1b_sound3_periodic_three_stage_checked.restype = i32
    handle.gm1b_psolver3_trajectory_checked.argtypes = [
        i32, i32, i32, pa, i32, f32, i32, f32, f32, f32, u32, u32, i32, vp, vp,
    ]
    handle.gm1b_psolver3_trajectory_checked.restype = i32
    handle.gm1b_step_status_fold.argtypes = [vp, vp, vp, vp]
    handle.gm1b_step_status_fold.restype = i32
    handle.gm1b_profiler_enable.argtypes = [i32]
    handle.gm1b_profiler_enable.restype = i32
    handle.gm1b_profiler_collect.argtypes = [ctypes.POINTER(KernelStat), i32, ctypes.POINTER(i32)]
    handle.gm1b_profiler_collect.restype = i32
    version = handle.gm1b_abi_version()
    if version != ABI_VERSION:
        raise RuntimeError(f"{LIB_PATH} has ABI {version}, this package needs {ABI_VERSION}")
    _lib = handle
    return handle


def check(status: int, what: str) -> None:
    if status != GM1B_OK:
        message = lib().gm1b_last_error().decode("utf-8", errors="replace")
        raise Gm1bError(f"{what} failed with status {status}: {message}")


def profiler_enable(on: bool) -> None:
    check(lib().gm1b_profiler_enable(1 if on else 0), "gm1b_profiler_enable")


def profiler_collect() -> list[dict]:
    """Per-kernel launches and total device ms recorded since the last call,
    sorted by total time (waits for the recorded events)."""
    cap = 64
    buf = (KernelStat * cap)()
    n = ctypes.c_int32()
    check(lib().gm1b_profiler_collect(buf, cap, ctypes.byref(n)), "gm1b_profiler_collect")
    return [
        {"name": buf[q].name.decode(), "launches": int(buf[q].launches), "total_ms": float(buf[q].total_ms)}
        for q in range(min(n.value, cap))
    ]
