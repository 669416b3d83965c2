"""TKE evolution on the terrain lane on B200: turbt and the RK stages.

Drop-in mirror of the reference operator API (torch CUDA tensors in place of
CuPy arrays; the same names, keywords, contracts and refusals):

  TkeEvolutionSelection, tke_evolution_shapes     src/cm1core/cuda_tke_evolution.py:66-122
  launch_cuda_tke_diffusion                       :421  (turbt, once per large step)
  launch_cuda_tke_rk_stage                        :430  (one stage into workspace, then tke3d)
  launch_cuda_tke_commit                          :445  (tkea = tke3d after stage 3)
  launch_cuda_tke_evolution_frozen_flux           :456  (all of it with one flux snapshot)
  launch_cuda_tke_evolution                       :481  (refused, as in the reference)
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, fields
from typing import Any, Mapping

import torch

from . import _native
from .errors import refuse
from .periodic import CudaLaunch

NGXY = 3
_STRUCT = ("tkea", "tke3d", "tketen", "kmh", "kmv", "rho", "rf", "mh", "mf", "gz", "rgz", "rgzu", "rgzv", "c1", "c2",
           "rrf0", "rru", "rrv", "rrw", "divx")


@dataclass(frozen=True, slots=True)
class TkeEvolutionSelection:
    terrain: bool = True
    axisymmetric: int = 0
    lateral_boundaries: tuple[int, int, int, int] = (2, 2, 2, 2)
    serial_full_domain: bool = True
    doimpl: int = 1
    scalar_horizontal_order: int = 5
    scalar_vertical_order: int = 5
    scalar_weno: int = 2
    weno_order: int = 5
    nrkmax: int = 3
    positive_definite: bool = False


DEFAULT_TKE_EVOLUTION_SELECTION = TkeEvolutionSelection()


def _validate_selection(selection: TkeEvolutionSelection) -> None:
    if not isinstance(selection, TkeEvolutionSelection):
        raise TypeError("selection must be a TkeEvolutionSelection")
    if selection != DEFAULT_TKE_EVOLUTION_SELECTION:
        refuse(code="CM1-TKE-EVOLUTION-UNSUPPORTED", gate="physics-seam", option="tke_evolution_selection",
               value={f.name: getattr(selection, f.name) for f in fields(selection)},
               reason="another value selects a different turbt, advw, boundary, or cadence branch",
               remedy="use the terrain-lane selection")


def _validate_grid(ni: int, nj: int, nk: int) -> None:
    for name, value, minimum in (("ni", ni, 7), ("nj", nj, 7), ("nk", nk, 8)):
        if isinstance(value, bool) or not isinstance(value, int) or value < minimum:
            raise ValueError(f"{name} must be an integer >= {minimum}")


def _spacing(name: str, value: Any) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise TypeError(f"{name} must be numeric")
    x = float(value)
    if not math.isfinite(x) or x <= 0.0:
        raise ValueError(f"{name} must be finite and > 0")
    return x


def tke_evolution_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    _validate_grid(ni, nj, nk)
    mass, face, ng = (nk, nj, ni), (nk + 1, nj, ni), NGXY
    return {"tkea": face, "tke3d": face, "tketen": face, "kmh": face, "kmv": face, "rho": mass, "rf": face,
            "mh": mass, "mf": face, "gz": (nj, ni), "rgz": (nj, ni), "rgzu": (nj, ni + 1), "rgzv": (nj + 1, ni),
            "c1": face, "c2": face, "rrf0": face, "rru": (nk + 2, nj + 2 * ng, ni + 1 + 2 * ng),
            "rrv": (nk + 2, nj + 1 + 2 * ng, ni + 2 * ng), "rrw": (nk + 3, nj + 2 * ng, ni + 2 * ng), "divx": mass}


class _Arrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in _STRUCT]


def _lib():
    lib = _native.lib()
    if not getattr(lib, "_tkeevo_bound", False):
        i32, f32, vp = ctypes.c_int32, ctypes.c_float, ctypes.c_void_p
        pa = ctypes.POINTER(_Arrays)
        lib.gm1b_tke_diffusion.argtypes = [i32, i32, i32, pa, f32, f32, f32, f32, vp]
        lib.gm1b_tke_diffusion.restype = i32
        lib.gm1b_tke_rk_stage.argtypes = [i32, i32, i32, pa, vp, vp, i32, f32, f32, f32, f32, vp]
        lib.gm1b_tke_rk_stage.restype = i32
        lib.gm1b_tke_evolution.argtypes = [i32, i32, i32, pa, vp, f32, f32, f32, f32, vp]
        lib.gm1b_tke_evolution.restype = i32
        lib.gm1b_tke_diffusion_flat.argtypes = [i32, i32, i32, pa, f32, f32, f32, f32, vp]
        lib.gm1b_tke_diffusion_flat.restype = i32
        lib.gm1b_tke_rk_stage_flat.argtypes = [i32, i32, i32, pa, vp, vp, vp, i32, f32, f32, f32, f32, vp]
        lib.gm1b_tke_rk_stage_flat.restype = i32
        lib._tkeevo_bound = True
    return lib


def _arrays(arrays: Mapping[str, Any], ni: int, nj: int, nk: int) -> dict[str, torch.Tensor]:
    shapes = tke_evolution_shapes(ni, nj, nk)
    missing = [n for n in _STRUCT if n not in arrays]
    if missing:
        raise ValueError(f"missing TKE evolution arrays: {', '.join(missing)}")
    out = {}
    for n in _STRUCT:
        t = arrays[n]
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 \
                or tuple(t.shape) != shapes[n] or not t.is_contiguous():
            raise ValueError(f"{n} must be a C-order float32 CUDA tensor with shape {shapes[n]}")
        out[n] = t
    if len({t.data_ptr() for t in out.values()}) != len(out):
        raise ValueError("TKE evolution arrays must not alias")
    return out


def _workspace(workspace: Any, a: dict[str, torch.Tensor], shape) -> torch.Tensor:
    if not isinstance(workspace, torch.Tensor) or not workspace.is_cuda or workspace.dtype != torch.float32 \
            or tuple(workspace.shape) != shape or not workspace.is_contiguous():
        raise ValueError(f"workspace must be a C-order float32 CUDA tensor with shape {shape}")
    if workspace.data_ptr() in {t.data_ptr() for t in a.values()}:
        raise ValueError("TKE stage workspace must not alias persistent arrays")
    return workspace


def _call(fn, *args) -> None:
    _native.check(fn(*args), fn.__name__)


def _launch(a, stream, body, receipt) -> CudaLaunch:
    device = a["tke3d"].device
    st = torch.cuda.current_stream(device) if stream is None else stream
    s = _Arrays(**{n: a[n].data_ptr() for n in _STRUCT})
    with torch.cuda.device(device), torch.cuda.stream(st):
        body(s, ctypes.c_void_p(st.cuda_stream))
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, receipt)


def launch_cuda_tke_diffusion(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float, dz: float,
                              dt: float, stream: Any | None = None,
                              selection: TkeEvolutionSelection = DEFAULT_TKE_EVOLUTION_SELECTION) -> CudaLaunch:
    """Apply turbt once (adds into tketen); do not call inside RK."""
    _validate_selection(selection)
    _validate_grid(ni, nj, nk)
    dx, dy, dz, dt = (_spacing(n, v) for n, v in (("dx", dx), ("dy", dy), ("dz", dz), ("dt", dt)))
    a = _arrays(arrays, ni, nj, nk)
    lib = _lib()
    return _launch(a, stream, lambda s, st: _call(lib.gm1b_tke_diffusion, ni, nj, nk, ctypes.byref(s), dx, dy, dz, dt,
                                                  st), {"phase": "solve1-turbt-once"})


def launch_cuda_tke_rk_stage(arrays: Mapping[str, Any], *, workspace: Any, ni: int, nj: int, nk: int, nrk: int,
                             dx: float, dy: float, dz: float, dt: float, stream: Any | None = None,
                             selection: TkeEvolutionSelection = DEFAULT_TKE_EVOLUTION_SELECTION) -> CudaLaunch:
    """One advw/RK stage from tke3d into workspace, then tke3d = workspace
    (tkea, the full-step baseline, is not modified)."""
    _validate_selection(selection)
    _validate_grid(ni, nj, nk)
    if isinstance(nrk, bool) or not isinstance(nrk, int) or nrk not in (1, 2, 3):
        raise ValueError("nrk must be an integer in 1..3")
    dx, dy, dz, dt = (_spacing(n, v) for n, v in (("dx", dx), ("dy", dy), ("dz", dz), ("dt", dt)))
    a = _arrays(arrays, ni, nj, nk)
    ws = _workspace(workspace, a, (nk + 1, nj, ni))
    lib = _lib()

    def body(s, st):
        _call(lib.gm1b_tke_rk_stage, ni, nj, nk, ctypes.byref(s), a["tke3d"].data_ptr(), ws.data_ptr(), nrk,
              dx, dy, dz, dt, st)
        a["tke3d"].copy_(ws)

    return _launch(a, stream, body, {"phase": "solve2-tke-advw-rk-stage", "nrk": nrk, "uses_weno": nrk == 3})


def launch_cuda_tke_commit(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, completed_nrk: int,
                           stream: Any | None = None,
                           selection: TkeEvolutionSelection = DEFAULT_TKE_EVOLUTION_SELECTION) -> CudaLaunch:
    """tkea = tke3d, only after RK stage three."""
    _validate_selection(selection)
    _validate_grid(ni, nj, nk)
    if completed_nrk != 3:
        raise ValueError("TKE commit requires completed_nrk=3")
    a = _arrays(arrays, ni, nj, nk)
    return _launch(a, stream, lambda s, st: a["tkea"].copy_(a["tke3d"]), {"phase": "solve3-tkea-commit"})


def launch_cuda_tke_evolution_frozen_flux(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float,
                                          dy: float, dz: float, dt: float, stream: Any | None = None,
                                          workspace: torch.Tensor | None = None,
                                          selection: TkeEvolutionSelection = DEFAULT_TKE_EVOLUTION_SELECTION,
                                          ) -> CudaLaunch:
    """turbt, the three stages with one flux snapshot, and the commit (the
    operator the reference's CPU twin computes)."""
    _validate_selection(selection)
    _validate_grid(ni, nj, nk)
    dx, dy, dz, dt = (_spacing(n, v) for n, v in (("dx", dx), ("dy", dy), ("dz", dz), ("dt", dt)))
    a = _arrays(arrays, ni, nj, nk)
    if workspace is None:
        workspace = torch.empty((nk + 1, nj, ni), dtype=torch.float32, device=a["tke3d"].device)
    ws = _workspace(workspace, a, (nk + 1, nj, ni))
    lib = _lib()
    return _launch(a, stream, lambda s, st: _call(lib.gm1b_tke_evolution, ni, nj, nk, ctypes.byref(s), ws.data_ptr(),
                                                  dx, dy, dz, dt, st),
                   {"phase": "turbt+3 stages+commit", "weno_stages": [3]})


def launch_cuda_tke_evolution(*args: Any, **kwargs: Any) -> CudaLaunch:
    """Refuse the cadence-ambiguous all-stage entry point, as the reference does."""
    del args, kwargs
    refuse(code="CM1-TKE-FLUX-CADENCE", gate="physics-seam", option="launch_cuda_tke_evolution",
           value="all-three-stages",
           reason="CM1 rebuilds rru/rrv/rrw/divx after each acoustic stage; one snapshot cannot represent an "
                  "evolved RK trajectory",
           remedy="call launch_cuda_tke_diffusion once, launch_cuda_tke_rk_stage after each nrk getdivx, then "
                  "launch_cuda_tke_commit")


# ------------------------------------------------------- flat column family

FLAT_TURBT_NAMES = ("tke3d", "kmh", "kmv", "rho", "rf", "mh", "mf", "tketen")
FLAT_STAGE_NAMES = ("tkea", "tke3d", "tketen", "c2", "rrf0", "rru", "rrv", "rrw", "divx")


def _flat_arrays(arrays: Mapping[str, Any], names, ni: int, nj: int, nk: int) -> dict[str, torch.Tensor]:
    shapes = tke_evolution_shapes(ni, nj, nk)
    missing = [n for n in names if n not in arrays]
    if missing:
        raise ValueError(f"missing flat TKE arrays: {', '.join(missing)}")
    out = {}
    for n in names:
        t = arrays[n]
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 \
                or tuple(t.shape) != shapes[n] or not t.is_contiguous():
            raise ValueError(f"{n} must be a C-order float32 CUDA tensor with shape {shapes[n]}")
        out[n] = t
    if len({t.data_ptr() for t in out.values()}) != len(out):
        raise ValueError("flat TKE arrays must not alias")
    return out


def _flat_struct(a: dict[str, torch.Tensor]) -> _Arrays:
    return _Arrays(**{n: (a[n].data_ptr() if n in a else None) for n in _STRUCT})


def launch_cuda_flat_tke_diffusion(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float,
                                   rdz: float, dt: float, stream: Any | None = None) -> CudaLaunch:
    """turbt on a flat (terrain_flag=.false.) stretched column
    (enqueue_flat_turbt, src/cm1core/cuda_gm1_flat_stretched_closure.py:631):
    the face fluxes without a terrain correction and the implicit diffusion
    with the coordinate's reference ``rdz`` and the 3-D mh/mf; adds into
    tketen.  ``arrays``: tke3d, kmh, kmv, rho, rf, mh, mf, tketen."""
    _validate_grid(ni, nj, nk)
    dx, dy, rdz, dt = (_spacing(n, v) for n, v in (("dx", dx), ("dy", dy), ("rdz", rdz), ("dt", dt)))
    a = _flat_arrays(arrays, FLAT_TURBT_NAMES, ni, nj, nk)
    lib = _lib()
    device = a["tke3d"].device
    st = torch.cuda.current_stream(device) if stream is None else stream
    s = _flat_struct(a)
    with torch.cuda.device(device):
        _call(lib.gm1b_tke_diffusion_flat, ni, nj, nk, ctypes.byref(s), dx, dy, rdz, dt,
              ctypes.c_void_p(st.cuda_stream))
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {"phase": "solve1-turbt-once", "column": "flat"})


def launch_cuda_flat_tke_rk_stage(arrays: Mapping[str, Any], *, mf_profile: Any, workspace: Any, ni: int, nj: int,
                                  nk: int, nrk: int, dx: float, dy: float, rdz: float, dt: float,
                                  stream: Any | None = None) -> CudaLaunch:
    """One advw/RK stage on a flat stretched column from tke3d into
    workspace, then tke3d = workspace (the flat branch of
    CartesianClosure.tke_rk, src/cm1core/cuda_cartesian_closure.py:1658-1663):
    vertical divergence with rdz*mf(k) (``mf_profile``, nk+3 words), the
    column's c2 and rrf0, no gz.  ``arrays``: tkea, tke3d, tketen, c2, rrf0,
    rru, rrv, rrw, divx."""
    _validate_grid(ni, nj, nk)
    if isinstance(nrk, bool) or not isinstance(nrk, int) or nrk not in (1, 2, 3):
        raise ValueError("nrk must be an integer in 1..3")
    dx, dy, rdz, dt = (_spacing(n, v) for n, v in (("dx", dx), ("dy", dy), ("rdz", rdz), ("dt", dt)))
    a = _flat_arrays(arrays, FLAT_STAGE_NAMES, ni, nj, nk)
    if not isinstance(mf_profile, torch.Tensor) or not mf_profile.is_cuda or mf_profile.dtype != torch.float32 \
            or tuple(mf_profile.shape) != (nk + 3,) or not mf_profile.is_contiguous():
        raise ValueError(f"mf_profile must be a C-order float32 CUDA tensor of shape ({nk + 3},)")
    ws = _workspace(workspace, a, (nk + 1, nj, ni))
    lib = _lib()
    device = a["tke3d"].device
    st = torch.cuda.current_stream(device) if stream is None else stream
    s = _flat_struct(a)
    with torch.cuda.device(device), torch.cuda.stream(st):
        _call(lib.gm1b_tke_rk_stage_flat, ni, nj, nk, ctypes.byref(s), mf_profile.data_ptr(), a["tke3d"].data_ptr(),
              ws.data_ptr(), nrk, dx, dy, rdz, dt, ctypes.c_void_p(st.cuda_stream))
        a["tke3d"].copy_(ws)
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {"phase": "solve2-tke-advw-rk-stage", "column": "flat", "nrk": nrk, "uses_weno": nrk == 3})
