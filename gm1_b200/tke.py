"""Deardorff SGS/TKE local algebra on B200.

Drop-in mirror of the reference operator API (torch CUDA tensors in place of
CuPy arrays; the same array names, shapes, keywords and refusals):

  SgsTkeSelection, sgs_constants_f32  src/cm1core/cuda_sgs_tke.py:48-208
  sgs_tke_array_shapes                src/cm1core/cuda_sgs_tke.py:139-143
  launch_cuda_sgs_tke                 src/cm1core/cuda_sgs_tke.py:637
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Any, Mapping

import torch

from . import _native
from .errors import refuse
from .periodic import CudaLaunch


@dataclass(frozen=True, slots=True)
class SgsTkeSelection:
    cm1setup: int = 1
    sgsmodel: int = 1
    tconfig: int = 1
    bbc: int = 1
    tbc: int = 1
    axisymmetric: int = 0
    horizturb: int = 0
    doimpl: int = 1


DEFAULT_SGS_TKE_SELECTION = SgsTkeSelection()
_EXPECTED = {
    "physics.cm1setup": ("cm1setup", 1),
    "physics.sgs_model": ("sgsmodel", 1),
    "physics.tke_length_scale": ("tconfig", 1),
    "boundaries.lower": ("bbc", 1),
    "boundaries.upper": ("tbc", 1),
    "grid.axisymmetric": ("axisymmetric", 0),
    "physics.horizontal_turbulence": ("horizturb", 0),
    "physics.vertical_implicit_diffusion": ("doimpl", 1),
}
INPUT_ARRAY_NAMES = ("ruh", "rvh", "rmf", "nm", "defv", "defh")
MUTABLE_ARRAY_NAMES = ("tkea", "tk", "grdscl", "rgrdscl", "lenscl", "dissten", "cme", "ce1", "ce2", "csm", "kmh",
                       "kmv", "khh", "khv", "tketen")
ALL_ARRAY_NAMES = INPUT_ARRAY_NAMES + MUTABLE_ARRAY_NAMES


def _validate_selection(selection: SgsTkeSelection) -> None:
    if not isinstance(selection, SgsTkeSelection):
        raise TypeError("selection must be an SgsTkeSelection")
    for option, (attribute, expected) in _EXPECTED.items():
        value = getattr(selection, attribute)
        if isinstance(value, bool) or not isinstance(value, int) or value != expected:
            refuse(code="CM1-SGS-TKE-UNSUPPORTED", gate="physics-seam", option=option, value=value,
                   reason=f"only {option}={expected} is built; another value selects different CM1 branches",
                   remedy="use the single-length-scale LES branch")


def sgs_tke_array_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    for name, value, minimum in (("ni", ni, 1), ("nj", nj, 1), ("nk", nk, 2)):
        if isinstance(value, bool) or not isinstance(value, int) or value < minimum:
            raise ValueError(f"{name} must be an integer >= {minimum}")
    cell = (nk + 1, nj, ni)
    return {"ruh": (ni,), "rvh": (nj,), **{n: cell for n in ALL_ARRAY_NAMES if n not in ("ruh", "rvh")}}


class _SgsArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ALL_ARRAY_NAMES + ("clip_count",)]


def _bind() -> ctypes.CDLL:
    lib = _native.lib()
    if not getattr(lib, "_sgs_bound", False):
        i32, f32 = ctypes.c_int32, ctypes.c_float
        lib.gm1b_sgs_tke.argtypes = [i32, i32, i32, ctypes.POINTER(_SgsArrays), f32, f32, f32, ctypes.c_void_p]
        lib.gm1b_sgs_tke.restype = i32
        lib._sgs_bound = True
    return lib


def launch_cuda_sgs_tke(
    arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float, dz: float,
    selection: SgsTkeSelection = DEFAULT_SGS_TKE_SELECTION, stream: Any | None = None,
    clip_count: torch.Tensor | None = None,
) -> CudaLaunch:
    """Enqueue the local SGS/TKE operator without host synchronisation.
    ``clip_count`` (one int32 word) receives the number of clipped TKE words."""
    _validate_selection(selection)
    shapes = sgs_tke_array_shapes(ni, nj, nk)
    for name, value in (("dx", dx), ("dy", dy), ("dz", dz)):
        if isinstance(value, bool) or not isinstance(value, (int, float)) or not math.isfinite(value) or value <= 0:
            raise ValueError(f"{name} must be finite and > 0")
    missing = [n for n in ALL_ARRAY_NAMES if n not in arrays]
    if missing:
        raise ValueError(f"missing SGS/TKE arrays: {', '.join(missing)}")
    a = {}
    for n in ALL_ARRAY_NAMES:
        t = arrays[n]
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 \
                or tuple(t.shape) != shapes[n] or not t.is_contiguous():
            raise ValueError(f"{n} must be a contiguous float32 CUDA tensor of shape {shapes[n]}")
        a[n] = t
    if clip_count is not None:
        if clip_count.dtype != torch.int32 or clip_count.numel() != 1:
            raise ValueError("clip_count must be one int32 word")
        a["clip_count"] = clip_count
    if len({t.data_ptr() for t in a.values()}) != len(a):
        raise ValueError("SGS/TKE arrays must not alias")
    s = _SgsArrays(**{n: t.data_ptr() for n, t in a.items()})
    device = a["tkea"].device
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        _native.check(_bind().gm1b_sgs_tke(ni, nj, nk, ctypes.byref(s), dx, dy, dz, ctypes.c_void_p(st.cuda_stream)),
                      "gm1b_sgs_tke")
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {"operator": "sgs-tke", "interior_words": ni * nj * (nk - 1)})
