"""eqtset=2 moist stage terms on B200.

Device counterpart of the stage-terms launch of the reference
(launch_cuda_eqtset2_stage_terms, src/cm1core/cuda_moist_stage_bridge.py:378,
cell algebra cpu_eqtset2_cell_f32 :62): moist buoyancy, theta-rho (thv), the
theta and pressure energy terms (thterm, ppterm) and piadv, with the
reference's array names and layouts.
"""

from __future__ import annotations

import ctypes
from typing import Any

import torch

from . import _native
from .periodic import CudaLaunch


class _Eqtset2Arrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("th0", "qv0", "pi0", "qc0", "qi0", "th3d", "q3d", "pp3d", "thv",
                                               "ppterm", "buoyancy", "thterm", "piadv")]


def _bind() -> ctypes.CDLL:
    lib = _native.lib()
    if not getattr(lib, "_bridge_bound", False):
        i32 = ctypes.c_int32
        lib.gm1b_eqtset2_stage_terms.argtypes = [i32, i32, i32, ctypes.POINTER(_Eqtset2Arrays), i32, ctypes.c_void_p]
        lib.gm1b_eqtset2_stage_terms.restype = i32
        lib._bridge_bound = True
    return lib


def _req(t: Any, name: str, shape: tuple[int, ...]) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 or tuple(t.shape) != shape \
            or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor of shape {shape}")
    return t


def launch_cuda_eqtset2_stage_terms(*, ni: int, nj: int, nk: int, th0, qv0, pi0, th3d, q3d, pp3d, thv, ppterm,
                                    buoyancy, thterm, piadv, qc0=None, qi0=None, base3d: bool = False,
                                    stream: Any | None = None) -> CudaLaunch:
    """Enqueue the eqtset=2 stage terms.  ``qc0``/``qi0`` None: base
    condensate exactly zero (the reference's default)."""
    base_shape = (nk, nj, ni) if base3d else (nk,)
    per = (nk + 2, nj + 2, ni + 2)
    arrays = {
        "th0": _req(th0, "th0", base_shape), "qv0": _req(qv0, "qv0", base_shape), "pi0": _req(pi0, "pi0", base_shape),
        "qc0": None if qc0 is None else _req(qc0, "qc0", base_shape),
        "qi0": None if qi0 is None else _req(qi0, "qi0", base_shape),
        "th3d": _req(th3d, "th3d", (nk, nj, ni)), "q3d": _req(q3d, "q3d", (6, nk, nj, ni)),
        "pp3d": _req(pp3d, "pp3d", per), "thv": _req(thv, "thv", per), "ppterm": _req(ppterm, "ppterm", per),
        "buoyancy": _req(buoyancy, "buoyancy", (nk + 2, nj + 6, ni + 6)), "thterm": _req(thterm, "thterm", (nk, nj, ni)),
        "piadv": _req(piadv, "piadv", per),
    }
    live = [t for t in arrays.values() if t is not None]
    if len({t.data_ptr() for t in live}) != len(live):
        raise ValueError("moist stage arrays must not alias")
    s = _Eqtset2Arrays(**{n: (t.data_ptr() if t is not None else None) for n, t in arrays.items()})
    device = th3d.device
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        _native.check(_bind().gm1b_eqtset2_stage_terms(ni, nj, nk, ctypes.byref(s), 1 if base3d else 0,
                                                       ctypes.c_void_p(st.cuda_stream)), "gm1b_eqtset2_stage_terms")
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {"operator": "eqtset2-stage-terms", "base3d": base3d})
