"""Scalar/moisture RK stage pieces on the padded (ng = 3) lane, on B200.

Device counterparts, with the same argument names and orders, of the
reference's CPU twins (src/cm1core/cuda_scalar_moist_rk.py):

  theta_transport_scalar          <- cpu_theta_transport_scalar_inplace (:255)
  compose_scalar_moist_rk_stage   <- cpu_compose_scalar_moist_rk_stage_inplace (:283)
  pdef_direction                  <- cpu_pdef_direction_inplace (:352)
  scalar_moist_rk_stage_timestep_f32 (:141), moisture_weps_f64 (:168),
  theta_weps_f64 (:238)

All arrays are torch CUDA float32 tensors; each call enqueues on ``stream``
(the current torch stream by default) and returns a launch record.
"""

from __future__ import annotations

import ctypes
from typing import Any

import numpy as np
import torch

from . import _native
from .periodic import CudaLaunch

CM1_SCALAR_MOIST_SPECIES = ("qv", "qc", "qr", "qi", "qs", "qg")
CM1_EPSILON_F32 = 1.0e-18
CM1_QMAG_F32 = (1.0e-2,) * 6
NG = 3


def scalar_moist_rk_stage_timestep_f32(dt: float, nrk: int) -> float:
    if nrk not in (1, 2, 3):
        raise ValueError("nrk must be one of 1, 2, 3")
    return float(np.float32(np.float32(dt) / np.float32(4 - nrk)))


def moisture_weps_f64(species: int, qmag: tuple[float, ...] = CM1_QMAG_F32) -> float:
    """weps = qmag(n) * epsilon in binary32 (solve2.F:1472)."""
    if isinstance(species, bool) or not isinstance(species, int):
        raise TypeError("species must be an integer")
    if species < 0 or species >= len(qmag):
        raise ValueError(f"species must index one of {len(qmag)} CM1 q3d scalars")
    return float(np.float32(np.float32(qmag[species]) * np.float32(CM1_EPSILON_F32)))


def theta_weps_f64() -> float:
    return float(np.float32(np.float32(10.0) * np.float32(CM1_EPSILON_F32)))


class _ComposeArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("theta_a", "theta_held", "theta_divterm", "theta_adv", "theta_cur",
                                               "q_a", "q_held", "q_adv", "q_cur")]


class _PdefArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("scalar_a", "scalar_padded", "rho0", "gz", "rgz", "mass_flux",
                                               "directional", "candidate")]


def _bind() -> ctypes.CDLL:
    lib = _native.lib()
    if not getattr(lib, "_rk_bound", False):
        i32, f32, vp = ctypes.c_int32, ctypes.c_float, ctypes.c_void_p
        lib.gm1b_theta_transport_pack.argtypes = [i32, i32, i32, vp, vp, vp, vp]
        lib.gm1b_theta_transport_pack.restype = i32
        lib.gm1b_scalar_moist_rk_compose.argtypes = [ctypes.c_size_t, i32, ctypes.POINTER(_ComposeArrays), i32, f32,
                                                     vp]
        lib.gm1b_scalar_moist_rk_compose.restype = i32
        lib.gm1b_pdef_direction.argtypes = [i32, i32, i32, ctypes.POINTER(_PdefArrays), i32, f32, f32, vp]
        lib.gm1b_pdef_direction.restype = i32
        lib._rk_bound = True
    return lib


def _f32(t: Any, name: str, shape: tuple[int, ...]) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 or tuple(t.shape) != shape \
            or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor of shape {shape}")
    return t


def _launch(device: torch.device, stream: Any | None, call) -> CudaLaunch:
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        call(ctypes.c_void_p(st.cuda_stream))
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {})


def theta_transport_scalar(th0, th3d, padded, *, ni: int, nj: int, nk: int, stream=None) -> CudaLaunch:
    """padded[k+1, j+3, i+3] = (th0[k] - 300) + th3d[k, j, i]."""
    _f32(th0, "th0", (nk,))
    _f32(th3d, "th3d", (nk, nj, ni))
    _f32(padded, "padded", (nk + 2, nj + 2 * NG, ni + 2 * NG))
    return _launch(th3d.device, stream, lambda s: _native.check(
        _bind().gm1b_theta_transport_pack(ni, nj, nk, th0.data_ptr(), th3d.data_ptr(), padded.data_ptr(), s),
        "gm1b_theta_transport_pack"))


def compose_scalar_moist_rk_stage(theta_a, moisture_a, theta_held, moisture_held, theta_divergence_term,
                                  theta_advection, moisture_advection, theta_current, moisture_current, *,
                                  nrk: int, dt: float, stream=None) -> CudaLaunch:
    """One A-anchored theta/moisture RK stage (species-major moisture)."""
    shape = tuple(theta_a.shape)
    qshape = tuple(moisture_a.shape)
    if len(shape) != 3 or len(qshape) != 4 or qshape[1:] != shape:
        raise ValueError("theta arrays are (nk, nj, ni) and moisture arrays (nq, nk, nj, ni)")
    t = [_f32(x, n, shape) for x, n in ((theta_a, "theta_a"), (theta_held, "theta_held"),
                                         (theta_divergence_term, "theta_divergence_term"),
                                         (theta_advection, "theta_advection"), (theta_current, "theta_current"))]
    q = [_f32(x, n, qshape) for x, n in ((moisture_a, "moisture_a"), (moisture_held, "moisture_held"),
                                          (moisture_advection, "moisture_advection"),
                                          (moisture_current, "moisture_current"))]
    if len({x.data_ptr() for x in t + q}) != len(t + q):
        raise ValueError("RK inputs and outputs must not alias")
    s = _ComposeArrays(*[x.data_ptr() for x in t], *[x.data_ptr() for x in q])
    cells = theta_a.numel()
    return _launch(theta_a.device, stream, lambda st: _native.check(
        _bind().gm1b_scalar_moist_rk_compose(cells, qshape[0], ctypes.byref(s), nrk, dt, st),
        "gm1b_scalar_moist_rk_compose"))


def pdef_direction(scalar_a, scalar_padded, rho0, gz, rgz, mass_flux, directional, candidate, *, axis: str,
                   dt: float, spacing: float, stream=None) -> CudaLaunch:
    """One pdef direction pass ("x", "y" or "z")."""
    if axis not in ("x", "y", "z"):
        raise ValueError("axis must be x, y, or z")
    nk, nj, ni = scalar_a.shape
    cell = (nk, nj, ni)
    flux_shapes = {"x": (nk + 2, nj + 2 * NG, ni + 1 + 2 * NG), "y": (nk + 2, nj + 1 + 2 * NG, ni + 2 * NG),
                   "z": (nk + 3, nj + 2 * NG, ni + 2 * NG)}
    arrs = [_f32(scalar_a, "scalar_a", cell), _f32(scalar_padded, "scalar_padded", (nk + 2, nj + 2 * NG, ni + 2 * NG)),
            _f32(rho0, "rho0", cell), _f32(gz, "gz", (nj, ni)), _f32(rgz, "rgz", (nj, ni)),
            _f32(mass_flux, "mass_flux", flux_shapes[axis]), _f32(directional, "directional", cell),
            _f32(candidate, "candidate", cell)]
    s = _PdefArrays(*[x.data_ptr() for x in arrs])
    ax = {"x": 0, "y": 1, "z": 2}[axis]
    return _launch(scalar_a.device, stream, lambda st: _native.check(
        _bind().gm1b_pdef_direction(ni, nj, nk, ctypes.byref(s), ax, dt, spacing, st), "gm1b_pdef_direction"))
