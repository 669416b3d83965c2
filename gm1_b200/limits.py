"""CM1's time-step limits and advective Courant number on B200.

Mirror of the reference functions (same names, keywords and errors), on
libgm1b.so:

  cm1_acoustic_small_step_limit_s     src/cm1core/gm1_runtime.py:249
  cm1_diagnostic_acoustic_substeps    src/cm1core/gm1_runtime.py:284
  cm1_advective_courant               src/cm1core/gm1_runtime.py:458
  advective_courant_number            src/cm1core/storm_diagnostics.py:249 (calccflquick),
                                      here over explicit device winds

The scalars are binary64 host arithmetic inside the library; the domain
Courant number is one CUDA reduction pass.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _native

CM1_PSOLVER3_ACOUSTIC_SPEED_M_S = 360.0
CM1_PSOLVER3_ACOUSTIC_COURANT = 0.60
CM1_MIN_ACOUSTIC_SUBSTEPS = 4
CM1_COURANT_STOP = 1.5


def _lib():
    lib = _native.lib()
    if not getattr(lib, "_limits_ready", False):
        d, i32, vp = ctypes.c_double, ctypes.c_int32, ctypes.c_void_p
        f = ctypes.c_float
        lib.gm1b_acoustic_small_step_limit.argtypes = [d, d]
        lib.gm1b_acoustic_small_step_limit.restype = d
        lib.gm1b_diagnostic_acoustic_substeps.argtypes = [d, d, d, ctypes.POINTER(i32)]
        lib.gm1b_diagnostic_acoustic_substeps.restype = i32
        lib.gm1b_advective_courant.argtypes = [d] * 7 + [ctypes.POINTER(d)]
        lib.gm1b_advective_courant.restype = i32
        lib.gm1b_courant_max.argtypes = [i32, i32, i32] + [vp] * 6 + [f, f, f, vp, vp, vp]
        lib.gm1b_courant_max.restype = i32
        lib._limits_ready = True
    return lib


def _numeric(name: str, value) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise TypeError(f"{name} must be numeric")
    return float(value)


def _positive(name: str, value) -> float:
    x = _numeric(name, value)
    if not math.isfinite(x) or x <= 0:
        raise ValueError(f"{name} must be finite and positive")
    return x


def cm1_acoustic_small_step_limit_s(*, dx_m: float, dy_m: float) -> float:
    dx, dy = _positive("dx_m", dx_m), _positive("dy_m", dy_m)
    return float(_lib().gm1b_acoustic_small_step_limit(dx, dy))


def cm1_diagnostic_acoustic_substeps(*, dt_s: float, dx_m: float, dy_m: float) -> int:
    dt = _positive("dt_s", dt_s)
    dx, dy = _positive("dx_m", dx_m), _positive("dy_m", dy_m)
    n = ctypes.c_int32()
    _native.check(_lib().gm1b_diagnostic_acoustic_substeps(dt, dx, dy, ctypes.byref(n)),
                  "gm1b_diagnostic_acoustic_substeps")
    return int(n.value)


def cm1_advective_courant(*, dt_s: float, dx_m: float, dy_m: float, dz_m: float, u_m_s: float, v_m_s: float,
                          w_m_s: float) -> float:
    dt = _positive("dt_s", dt_s)
    dx, dy, dz = _positive("dx_m", dx_m), _positive("dy_m", dy_m), _positive("dz_m", dz_m)
    winds = []
    for name, value in (("u_m_s", u_m_s), ("v_m_s", v_m_s), ("w_m_s", w_m_s)):
        x = _numeric(name, value)
        if not math.isfinite(x):
            raise ValueError(f"{name} must be finite")
        winds.append(x)
    out = ctypes.c_double()
    _native.check(_lib().gm1b_advective_courant(dt, dx, dy, dz, *winds, ctypes.byref(out)), "gm1b_advective_courant")
    return float(out.value)


def courant_factors(*, dt_s: float, dx_m: float, dy_m: float, dz_m: float) -> tuple[float, float, float]:
    """dtdx, dtdy, dtdz as binary32 in CM1's order: 0.5*dt*rdx with rdx the
    binary32 rounding of 1/dx (storm_diagnostics.py:278-280)."""
    f = np.float32
    dt = f(dt_s)
    return tuple(float(f(f(f(0.5) * dt) * f(1.0 / d))) for d in (dx_m, dy_m, dz_m))


def advective_courant_number(*, u: torch.Tensor, v: torch.Tensor, w: torch.Tensor, uh: torch.Tensor,
                             vh: torch.Tensor, mh: torch.Tensor, dt_s: float, dx_m: float, dy_m: float, dz_m: float,
                             level_keys: torch.Tensor | None = None, stream: torch.cuda.Stream | None = None,
                             out: torch.Tensor | None = None) -> torch.Tensor:
    """calccflquick over device winds u (nk, nj, ni+1), v (nk, nj+1, ni),
    w (nk+1, nj, ni); returns a one-word device tensor (no host sync)."""
    nk, nj, ni1 = u.shape
    ni = ni1 - 1
    shapes = {"u": (nk, nj, ni + 1), "v": (nk, nj + 1, ni), "w": (nk + 1, nj, ni), "uh": (ni,), "vh": (nj,),
              "mh": (nk,)}
    for name, t in (("u", u), ("v", v), ("w", w), ("uh", uh), ("vh", vh), ("mh", mh)):
        if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and tuple(t.shape) == shapes[name]):
            raise ValueError(f"{name} must be a contiguous float32 CUDA tensor of shape {shapes[name]}")
    dtdx, dtdy, dtdz = courant_factors(dt_s=dt_s, dx_m=dx_m, dy_m=dy_m, dz_m=dz_m)
    if level_keys is None:
        level_keys = torch.empty(nk, dtype=torch.int32, device=u.device)
    if out is None:
        out = torch.empty(1, dtype=torch.float32, device=u.device)
    st = stream if stream is not None else torch.cuda.current_stream(u.device)
    _native.check(_lib().gm1b_courant_max(ni, nj, nk, u.data_ptr(), v.data_ptr(), w.data_ptr(), uh.data_ptr(),
                                          vh.data_ptr(), mh.data_ptr(), dtdx, dtdy, dtdz, level_keys.data_ptr(),
                                          out.data_ptr(), st.cuda_stream), "gm1b_courant_max")
    return out
