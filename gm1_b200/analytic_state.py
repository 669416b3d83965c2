"""Analytic initial state of the moist storm configurations.

Mirror of the reference's binary32 initializer (same names, argument meaning
and refusals), on libgm1b.so:

  weisman_klemp_column / _with_iterations   rust/cm1-state/src/storm_initialization.rs:187,194
  WeismanKlempSurface.official              rust/cm1-state/src/storm_initialization.rs:67-80
  analytic_shear_u / analytic_shear_v       rust/cm1-state/src/storm_initialization.rs:354,373
  build_theta_perturbation (iinit=1)        rust/cm1-state/src/initial_perturbation.rs:425,449-466

The base column (nk words, computed once) is host arithmetic inside the
library; the bubble field is written by a CUDA kernel straight into a device
scalar lane.  There is no Python or NumPy fallback.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _native

WK_HYDROSTATIC_ITERATIONS = 20
WK_QV_PBL = np.float32(0.014)

_F = ctypes.POINTER(ctypes.c_float)


def _lib():
    lib = _native.lib()
    if not getattr(lib, "_analytic_ready", False):
        i32, f32, vp = ctypes.c_int32, ctypes.c_float, ctypes.c_void_p
        lib.gm1b_wk_base_column.argtypes = [i32, _F, i32, i32, _F, _F, _F, _F, _F, _F, _F]
        lib.gm1b_wk_base_column.restype = i32
        lib.gm1b_analytic_shear.argtypes = [i32, _F, _F, _F, _F]
        lib.gm1b_analytic_shear.restype = i32
        lib.gm1b_theta_bubble.argtypes = [i32, i32, i32, i32, vp, vp, vp, f32, f32, f32, f32, f32, f32, vp, vp]
        lib.gm1b_theta_bubble.restype = i32
        lib._analytic_ready = True
    return lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_F)


def _argument_error(status: int, what: str) -> None:
    if status == _native.GM1B_ERR_ARGUMENT:
        raise ValueError(_native.lib().gm1b_last_error().decode("utf-8", errors="replace"))
    _native.check(status, what)


@dataclass(frozen=True)
class WeismanKlempColumn:
    """One isnd=5 base column on the caller's mass heights (binary32)."""

    heights_m: np.ndarray
    theta_k: np.ndarray
    relative_humidity: np.ndarray
    qv_kg_per_kg: np.ndarray
    theta_v_k: np.ndarray
    pi: np.ndarray
    pressure_pa: np.ndarray
    temperature_k: np.ndarray
    iterations: int
    imoist: int

    def surface_qv_kg_per_kg(self, weights) -> np.float32:
        """base.F:442-450 with CM1's cgs1..cgs3 bottom extrapolation weights
        (storm_initialization.rs:166-182)."""
        if self.imoist != 1:
            return np.float32(0.0)
        if self.qv_kg_per_kg.size < 3:
            raise ValueError("analytic surface qv needs the lowest three mass levels (base.F:444)")
        q = self.qv_kg_per_kg
        w = np.asarray(weights, dtype=np.float32)
        if q[0] < WK_QV_PBL:
            return np.float32(np.float32(w[0] * q[0]) + np.float32(w[1] * q[1])) + np.float32(w[2] * q[2])
        return WK_QV_PBL


def weisman_klemp_column_with_iterations(heights_m, imoist: int, iterations: int) -> WeismanKlempColumn:
    z = np.ascontiguousarray(np.asarray(heights_m, dtype=np.float32))
    if z.ndim != 1:
        raise ValueError("analytic sounding heights must be one column")
    if isinstance(imoist, bool) or not isinstance(imoist, (int, np.integer)):
        raise TypeError("imoist must be an integer")
    nk = int(z.size)
    out = {n: np.zeros(max(nk, 1), np.float32) for n in ("th0", "qv0", "thv0", "pi0", "prs0", "t0", "rh0")}
    status = _lib().gm1b_wk_base_column(nk, _ptr(z) if nk else None, int(imoist), int(iterations),
                                        *(_ptr(out[n]) for n in ("th0", "qv0", "thv0", "pi0", "prs0", "t0", "rh0")))
    _argument_error(status, "gm1b_wk_base_column")
    return WeismanKlempColumn(heights_m=z.copy(), theta_k=out["th0"], relative_humidity=out["rh0"],
                              qv_kg_per_kg=out["qv0"], theta_v_k=out["thv0"], pi=out["pi0"],
                              pressure_pa=out["prs0"], temperature_k=out["t0"], iterations=int(iterations),
                              imoist=int(imoist))


def weisman_klemp_column(heights_m, imoist: int) -> WeismanKlempColumn:
    """The isnd=5 column with CM1's exact 20 hydrostatic iterations."""
    return weisman_klemp_column_with_iterations(heights_m, imoist, WK_HYDROSTATIC_ITERATIONS)


def _shear(z, which: str) -> np.ndarray:
    zz = np.ascontiguousarray(np.atleast_1d(np.asarray(z, dtype=np.float32)))
    out = np.zeros(zz.shape, np.float32)
    u = _ptr(out) if which == "u" else None
    v = _ptr(out) if which == "v" else None
    _native.check(_lib().gm1b_analytic_shear(int(zz.size), _ptr(zz), _ptr(zz), u, v), "gm1b_analytic_shear")
    return out


def analytic_shear_u(zu_m) -> np.ndarray:
    """iwnd=2 u0 on u-face heights (base.F:2331-2339), vectorised."""
    return _shear(zu_m, "u")


def analytic_shear_v(zv_m) -> np.ndarray:
    """iwnd=2 v0 on v-face heights (base.F:2344-2357), vectorised."""
    return _shear(zv_m, "v")


@dataclass(frozen=True)
class WarmBubbleControls:
    """iinit=1 bubble controls (init3d.F namelist words ric, rjc, zc, bhrad,
    bzrad, bptpert as the reference names them)."""

    center_x_m: float
    center_y_m: float
    center_z_agl_m: float
    horizontal_radius_m: float
    vertical_radius_m: float
    amplitude_k: float


def build_theta_perturbation(tha: torch.Tensor, controls: WarmBubbleControls, *, xh: torch.Tensor,
                             yh: torch.Tensor, zh: torch.Tensor, ni: int, nj: int, nk: int, ng: int,
                             stream: torch.cuda.Stream | None = None) -> None:
    """Write the iinit=1 cos^2 bubble into the interior of the device scalar
    lane ``tha`` (ng = 0 dense, 1 periodic lane, 3 padded lane)."""
    gz = 1 if ng > 0 else 0
    shape = (nk + 2 * gz, nj + 2 * ng, ni + 2 * ng)
    for name, t, n in (("xh", xh, ni), ("yh", yh, nj), ("zh", zh, nk)):
        if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and t.numel() == n):
            raise ValueError(f"{name} must be a contiguous float32 CUDA tensor of {n} words")
    if not (tha.is_cuda and tha.dtype == torch.float32 and tha.is_contiguous() and tuple(tha.shape) == shape):
        raise ValueError(f"tha must be a contiguous float32 CUDA tensor of shape {shape}")
    st = stream if stream is not None else torch.cuda.current_stream(tha.device)
    status = _lib().gm1b_theta_bubble(
        ni, nj, nk, ng, xh.data_ptr(), yh.data_ptr(), zh.data_ptr(), controls.center_x_m, controls.center_y_m,
        controls.center_z_agl_m, controls.horizontal_radius_m, controls.vertical_radius_m, controls.amplitude_k,
        tha.data_ptr(), st.cuda_stream)
    _argument_error(status, "gm1b_theta_bubble")
