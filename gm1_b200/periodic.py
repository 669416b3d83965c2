"""Operator API of the flat serial-periodic dry lane on B200.

Drop-in mirrors of the reference launchers, with torch CUDA tensors in place
of CuPy arrays (the dictionary keys, shapes, keyword arguments and error
behaviour are the reference's):

  launch_cuda_sound3_periodic_three_stage  src/cm1core/cuda_sound3_periodic.py:1216
  launch_cuda_psolver3_trajectory          src/cm1core/cuda_psolver3_trajectory.py:1460

Each call validates its arguments on the host, enqueues the CUDA kernels of
libgm1b.so on ``stream`` (the current torch stream by default) and returns a
launch record whose ``ready_event`` completes with the last kernel.  Nothing
is allocated on the device but a one-word status.  A stage that runs as the
one persistent kernel waits at a bounded grid barrier each small step; the
launch record's ``check()`` raises BarrierTimeout if one gave up, and the
launchers call it before they return (check_status=True, the default)
unless the stream is being captured into a CUDA graph, where the caller
calls ``check()`` after the replay.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, fields
from typing import Any, Mapping

import numpy as np
import torch

from . import _native
from .arrays import (
    ALL_ARRAY_NAMES,
    SOUND_ARRAY_NAMES,
    array_shapes,
    trajectory_array_shapes,
)

CM1_SOUND3_PERIODIC_ALPH_F32 = 0.60
CM1_SOUND3_PERIODIC_KDIV_F32 = 0.10
CM1_SOUND3_PERIODIC_CP_F32 = 1005.7


@dataclass(frozen=True, slots=True)
class TrajectoryAblations:
    """Which terms of the dry trajectory run (all by default); the field names
    are those of the reference (src/cm1core/cuda_psolver3_trajectory.py:429-436)."""

    momentum_advection: bool = True
    scalar_advection: bool = True
    base_theta_advection: bool = True
    buoyancy: bool = True
    post_step_ppx: bool = True
    carrier_promotion: bool = True

    def mask(self) -> int:
        m = 0
        for f in fields(self):
            if not getattr(self, f.name):
                m |= _native.ABLATION_BITS[f.name]
        return m


@dataclass(frozen=True)
class CudaLaunch:
    ready_event: torch.cuda.Event
    receipt: dict[str, Any]
    # one device int32: 1 once a persistent acoustic stage's grid barrier gave
    # up (its fields are then invalid), else 0
    barrier_status: torch.Tensor | None = None

    def check(self) -> None:
        """Wait for the launch and raise if a persistent acoustic stage's
        grid barrier gave up (the reference reads its device status words
        back and refuses in the same way, src/cm1core/cuda_graphs.py:197)."""
        self.ready_event.synchronize()
        if self.barrier_status is not None and int(self.barrier_status.item()) != 0:
            raise BarrierTimeout("a persistent acoustic stage's grid barrier gave up waiting for its CTAs; "
                                 "the fields of this launch are invalid")


class BarrierTimeout(_native.Gm1bError):
    """A persistent acoustic stage's bounded grid barrier ran out."""


def sound3_stage_schedule_f32(dt: float, nsound: int, nrk: int) -> tuple[int, float]:
    """(nloop, dts) of one RK stage, computed by the library
    (src/cm1core/cuda_sound3_column.py:391-417)."""
    if isinstance(nsound, bool) or not isinstance(nsound, int) or nsound < 4:
        raise ValueError("nsound must be an integer >= 4")
    if nsound % 2:
        raise ValueError("native diagnostic cadence requires even nsound")
    if isinstance(nrk, bool) or not isinstance(nrk, int) or nrk not in (1, 2, 3):
        raise ValueError("nrk must be one of 1, 2, 3")
    n = ctypes.c_int32()
    d = ctypes.c_float()
    _native.check(
        _native.lib().gm1b_sound3_stage_schedule(dt, nsound, nrk, ctypes.byref(n), ctypes.byref(d)),
        "gm1b_sound3_stage_schedule",
    )
    return int(n.value), float(d.value)


def rk_stage_dt_f32(dt: float, nrk: int) -> float:
    if nrk not in (1, 2, 3):
        raise ValueError("nrk must be one of 1, 2, 3")
    return float(_native.lib().gm1b_rk_stage_dt(dt, nrk))


def _require_device_arrays(
    arrays: Mapping[str, Any], names: tuple[str, ...], shapes: dict[str, tuple[int, ...]], what: str
) -> tuple[dict[str, torch.Tensor], torch.device]:
    missing = [name for name in names if name not in arrays]
    if missing:
        raise ValueError(f"missing {what} arrays: {', '.join(missing)}")
    result: dict[str, torch.Tensor] = {}
    device = None
    for name in names:
        value = arrays[name]
        if not isinstance(value, torch.Tensor):
            raise TypeError(f"{name} must be a torch.Tensor")
        if not value.is_cuda:
            raise ValueError(f"{name} must be a CUDA tensor")
        if value.dtype != torch.float32 or tuple(value.shape) != shapes[name] or not value.is_contiguous():
            raise ValueError(f"{name} has invalid CUDA dtype, shape, or layout")
        if device is None:
            device = value.device
        elif value.device != device:
            raise ValueError(f"{name} is on {value.device}, expected {device}")
        result[name] = value
    if len({t.data_ptr() for t in result.values()}) != len(result):
        raise ValueError(f"{what} device arrays must not alias")
    return result, device


def _struct(a: Mapping[str, torch.Tensor]) -> _native.PeriodicArrays:
    s = _native.PeriodicArrays()
    for name in ALL_ARRAY_NAMES:
        if name in a:
            setattr(s, name, a[name].data_ptr())
    return s


def _stream(stream: Any | None, device: torch.device) -> torch.cuda.Stream:
    return torch.cuda.current_stream(device) if stream is None else stream


def launch_cuda_sound3_periodic_three_stage(
    arrays: Mapping[str, Any],
    *,
    ni: int,
    nj: int,
    nk: int,
    dt: float,
    nsound: int,
    rdx: float,
    rdy: float,
    rdz: float,
    cp: float = CM1_SOUND3_PERIODIC_CP_F32,
    alph: float = CM1_SOUND3_PERIODIC_ALPH_F32,
    kdiv: float = CM1_SOUND3_PERIODIC_KDIV_F32,
    stream: Any | None = None,
    scratch_outputs: bool = False,
    fused_stage: bool = True,
    barrier_spin_limit: int = 0,
    check_status: bool = True,
) -> CudaLaunch:
    """Enqueue the three periodic acoustic RK stages.

    ``barrier_spin_limit`` bounds the persistent stage's barrier waits in
    polls (0: the library's default of about a second).

    ``scratch_outputs`` also writes the reference-semantics scratch arrays of
    the last small step (fpk, divh, hadvp, elim_c, elim_d, tri_*); without it
    those arrays are left unspecified.  ``fused_stage`` lets a stage without
    scratch outputs run as one persistent kernel (same words); False forces
    two launches per small step."""
    for nrk in (1, 2, 3):
        sound3_stage_schedule_f32(dt, nsound, nrk)
    a, device = _require_device_arrays(arrays, SOUND_ARRAY_NAMES, array_shapes(ni, nj, nk), "periodic sound3")
    st = _stream(stream, device)
    s = _struct(a)
    flags = _native.GM1B_FLAG_SCRATCH_OUTPUTS if scratch_outputs else 0
    if not fused_stage:
        flags |= _native.GM1B_FLAG_MULTI_LAUNCH_STAGE
    spin = _spin_limit(barrier_spin_limit)
    with torch.cuda.device(device):
        word = torch.zeros(1, dtype=torch.int32, device=device)
        status = _native.lib().gm1b_sound3_periodic_three_stage_checked(
            ni, nj, nk, ctypes.byref(s), dt, nsound, rdx, rdy, rdz, cp, alph, kdiv, flags, spin,
            ctypes.c_void_p(word.data_ptr()), ctypes.c_void_p(st.cuda_stream),
        )
        _native.check(status, "gm1b_sound3_periodic_three_stage")
        event = torch.cuda.Event()
        event.record(st)
    cadence = []
    for nrk in (1, 2, 3):
        nloop, dts = sound3_stage_schedule_f32(dt, nsound, nrk)
        cadence.append({"nrk": nrk, "nloop": nloop, "dts_f32": dts, "dttmp_f32": rk_stage_dt_f32(dt, nrk)})
    launch = CudaLaunch(event, {"operator": "sound3_periodic_three_stage", "cadence": cadence}, word)
    _maybe_check(launch, st, check_status)
    return launch


def _spin_limit(value: Any) -> int:
    if isinstance(value, bool) or not isinstance(value, int) or value < 0 or value > 2**31 - 1:
        raise ValueError("barrier_spin_limit must be an integer in [0, 2**31)")
    return value


def _maybe_check(launch: CudaLaunch, st: torch.cuda.Stream, check_status: bool) -> None:
    if check_status and not torch.cuda.is_current_stream_capturing():
        launch.check()


def _validate_run_parameters(*, ni, nj, nk, dt, nsound, dx, dy, dz) -> None:
    if ni < 5 or nj < 5 or nk < 6:
        raise ValueError("fifth-order trajectory requires ni >= 5, nj >= 5, nk >= 6")
    for name, value in (("dt", dt), ("dx", dx), ("dy", dy), ("dz", dz)):
        value32 = np.float32(value)
        if not bool(np.isfinite(value32)) or not bool(value32 > np.float32(0.0)):
            raise ValueError(f"{name} must be finite and positive in float32")
    for nrk in (1, 2, 3):
        sound3_stage_schedule_f32(dt, nsound, nrk)


def launch_cuda_psolver3_trajectory(
    arrays: Mapping[str, Any],
    *,
    ni: int,
    nj: int,
    nk: int,
    steps: int,
    dt: float,
    nsound: int,
    dx: float,
    dy: float,
    dz: float,
    ablations: TrajectoryAblations | int | None = None,
    stream: Any | None = None,
    scratch_outputs: bool = True,
    fused_stage: bool = True,
    barrier_spin_limit: int = 0,
    check_status: bool = True,
) -> CudaLaunch:
    """Enqueue ``steps`` dry RK3 large steps of the periodic trajectory.

    ``scratch_outputs`` (default, as the reference's outputs include them)
    writes tri_pivot/tri_residual and the other acoustic scratch arrays of the
    final small step; pass False for the fastest path, where each acoustic
    stage runs as one persistent kernel unless ``fused_stage`` is False."""
    if isinstance(steps, bool) or not isinstance(steps, int) or steps < 1:
        raise ValueError("steps must be an integer >= 1")
    _validate_run_parameters(ni=ni, nj=nj, nk=nk, dt=dt, nsound=nsound, dx=dx, dy=dy, dz=dz)
    a, device = _require_device_arrays(arrays, ALL_ARRAY_NAMES, trajectory_array_shapes(ni, nj, nk),
                                       "psolver3 trajectory")
    if ablations is None:
        mask = 0
    elif isinstance(ablations, int):
        mask = ablations
    else:
        mask = TrajectoryAblations(**{f.name: getattr(ablations, f.name) for f in fields(TrajectoryAblations)}).mask()
    st = _stream(stream, device)
    s = _struct(a)
    flags = _native.GM1B_FLAG_SCRATCH_OUTPUTS if scratch_outputs else 0
    if not fused_stage:
        flags |= _native.GM1B_FLAG_MULTI_LAUNCH_STAGE
    spin = _spin_limit(barrier_spin_limit)
    with torch.cuda.device(device):
        word = torch.zeros(1, dtype=torch.int32, device=device)
        status = _native.lib().gm1b_psolver3_trajectory_checked(
            ni, nj, nk, ctypes.byref(s), steps, dt, nsound, dx, dy, dz, mask, flags, spin,
            ctypes.c_void_p(word.data_ptr()), ctypes.c_void_p(st.cuda_stream),
        )
        _native.check(status, "gm1b_psolver3_trajectory")
        event = torch.cuda.Event()
        event.record(st)
    cadence = []
    for nrk in (1, 2, 3):
        nloop, dts = sound3_stage_schedule_f32(dt, nsound, nrk)
        cadence.append({"nrk": nrk, "nloop": nloop, "dts_f32": dts, "dttmp_f32": rk_stage_dt_f32(dt, nrk)})
    receipt = {
        "operator": "psolver3_trajectory",
        "steps": steps,
        "cadence": cadence,
        "ablation_mask": mask,
        "cells": ni * nj * nk,
    }
    launch = CudaLaunch(event, receipt, word)
    _maybe_check(launch, st, check_status)
    return launch


def to_device(arrays: Mapping[str, np.ndarray], device: str | torch.device = "cuda") -> dict[str, torch.Tensor]:
    """Copy a dictionary of host arrays to fresh contiguous device tensors."""
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(device) for k, v in arrays.items()}


def to_host(arrays: Mapping[str, torch.Tensor]) -> dict[str, np.ndarray]:
    return {k: v.detach().cpu().numpy() for k, v in arrays.items()}
