"""Device pieces that join the operators of the moist large step (torch
CUDA tensors; every call enqueues on ``stream``, the current stream by
default, and synchronises nothing):

  open_fill             cpu_bcp/bcs/bcu/bcv/bcw_open_inplace
                        (src/cm1core/cuda_sound3_open_boundary.py:249-335)
  moist_buoyancy        launch_cuda_moist_buoyancy (src/cm1core/cuda_moist_stage_bridge.py:433)
  post_acoustic_flux    launch_cuda_post_acoustic_flux_bridge (:461)
  pdef_moisture_chain   the final-stage moisture chain of launch_cuda_scalar_moist_rk_stage
                        (src/cm1core/cuda_scalar_moist_rk.py:1336-1500)
  held_compose          gm1_child_predict_and_compose_held_base3d_v1
                        (src/cm1core/cuda_gm1_child_step_composer.py:547)
  solve3_density        gm1_solve3_density_v1 (src/cm1core/cuda_gm1_forecast.py:548)
  pack_scalar           cm1_rk_pack_scalar_v1
"""

from __future__ import annotations

import ctypes
from typing import Any, Mapping

import torch

from . import _native
from .advection import StretchedColumn, _VerticalColumn

FILL_KINDS = {"pressure": 0, "scalar": 1, "u": 2, "v": 3, "w": 4, "w_keep_ends": 5}
POST_NAMES = ("rru", "rrv", "rrw", "rgzu", "rgzv", "dzdx", "dzdy", "gz", "rho0_3d", "rf0", "thterm", "divergence",
              "theta_divergence_term", "divx")
CHAIN_NAMES = ("scalar_a", "scalar_padded", "rho0_3d", "gz", "rgz", "rr0", "c1", "c2", "divx", "rru", "rrv", "rrw",
               "fx", "fy", "fz", "advx", "advy", "advz", "candidate", "advection")
HELD_NAMES = ("th0", "pi0", "rho", "ppi", "tha", "qa", "qpten", "qtten", "qvten", "qcten", "thheld", "qheld", "ppten")


def _struct(names):
    class S(ctypes.Structure):
        _fields_ = [(n, ctypes.c_void_p) for n in names]
    return S


_Post, _Chain, _Held = _struct(POST_NAMES), _struct(CHAIN_NAMES), _struct(HELD_NAMES)


def _lib():
    lib = _native.lib()
    if not getattr(lib, "_mops_bound", False):
        c = ctypes
        i, f, vp = c.c_int32, c.c_float, c.c_void_p
        lib.gm1b_open_fill.argtypes = [i, i, i, i, vp, vp]
        lib.gm1b_moist_buoyancy.argtypes = [i, i, i] + [vp] * 8 + [vp]
        lib.gm1b_post_acoustic_flux.argtypes = [i, i, i, c.POINTER(_Post), f, f, f, vp]
        lib.gm1b_pdef_moisture_chain.argtypes = [i, i, i, c.POINTER(_Chain), f, f, f, f, c.c_double, c.c_uint32, i, vp]
        lib.gm1b_pdef_moisture_chain_column.argtypes = [i, i, i, c.POINTER(_Chain), f, f, f, c.c_double, c.c_uint32,
                                                        i, c.POINTER(_VerticalColumn), vp]
        lib.gm1b_pdef_moisture_chain_column.restype = i
        from .momentum import _Column  # noqa: PLC0415

        lib.gm1b_post_acoustic_flux_column.argtypes = [i, i, i, c.POINTER(_Post), f, f, c.POINTER(_Column), vp]
        lib.gm1b_post_acoustic_flux_column.restype = i
        lib.gm1b_moist_buoyancy_flat.argtypes = [i, i, i] + [vp] * 4 + [vp]
        lib.gm1b_moist_buoyancy_flat.restype = i
        lib.gm1b_held_compose.argtypes = [i, i, i, c.POINTER(_Held), f, vp]
        lib.gm1b_solve3_density.argtypes = [i, i, i] + [vp] * 5 + [vp]
        lib.gm1b_pack_scalar.argtypes = [i, i, i, vp, vp, vp]
        lib.gm1b_bcwsfc.argtypes = [i, i, i] + [vp] * 7
        lib.gm1b_w_level1_fill.argtypes = [i, i, i, vp, vp]
        for n in ("gm1b_bcwsfc", "gm1b_w_level1_fill", "gm1b_open_fill", "gm1b_moist_buoyancy", "gm1b_post_acoustic_flux", "gm1b_pdef_moisture_chain",
                  "gm1b_held_compose", "gm1b_solve3_density", "gm1b_pack_scalar"):
            getattr(lib, n).restype = i
        lib._mops_bound = True
    return lib


def _f32(t: Any, name: str) -> int:
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor")
    return t.data_ptr()


def _st(stream, device) -> ctypes.c_void_p:
    st = torch.cuda.current_stream(device) if stream is None else stream
    return ctypes.c_void_p(st.cuda_stream)


def open_fill(q: torch.Tensor, kind: str, *, ni: int, nj: int, nk: int, stream: Any | None = None) -> None:
    if kind not in FILL_KINDS:
        raise ValueError(f"kind must be one of {tuple(FILL_KINDS)}")
    _native.check(_lib().gm1b_open_fill(ni, nj, nk, FILL_KINDS[kind], _f32(q, "q"), _st(stream, q.device)),
                  "gm1b_open_fill")


def moist_buoyancy(dum8, c1, c2, gxu, gyv, uten, vten, wten, *, ni: int, nj: int, nk: int,
                   stream: Any | None = None) -> None:
    ptrs = [_f32(t, n) for t, n in zip((dum8, c1, c2, gxu, gyv, uten, vten, wten),
                                       ("dum8", "c1", "c2", "gxu", "gyv", "uten", "vten", "wten"))]
    _native.check(_lib().gm1b_moist_buoyancy(ni, nj, nk, *ptrs, _st(stream, dum8.device)), "gm1b_moist_buoyancy")


def post_acoustic_flux(a: Mapping[str, torch.Tensor], *, ni: int, nj: int, nk: int, dx: float, dy: float, dz: float,
                       stream: Any | None = None) -> None:
    s = _Post(**{n: _f32(a[n], n) for n in POST_NAMES})
    _native.check(_lib().gm1b_post_acoustic_flux(ni, nj, nk, ctypes.byref(s), dx, dy, dz, _st(stream, a["rru"].device)),
                  "gm1b_post_acoustic_flux")


def pdef_moisture_chain(a: Mapping[str, torch.Tensor], *, ni: int, nj: int, nk: int, dttmp: float, dx: float,
                        dy: float, dz: float, weps: float, lateral_obc: int, pdefweno: int,
                        stream: Any | None = None) -> None:
    s = _Chain(**{n: _f32(a[n], n) for n in CHAIN_NAMES})
    _native.check(_lib().gm1b_pdef_moisture_chain(ni, nj, nk, ctypes.byref(s), dttmp, dx, dy, dz, weps, lateral_obc,
                                                  pdefweno, _st(stream, a["rru"].device)), "gm1b_pdef_moisture_chain")


def pdef_moisture_chain_column(a: Mapping[str, torch.Tensor], column: StretchedColumn, *, ni: int, nj: int, nk: int,
                               dttmp: float, dx: float, dy: float, weps: float, lateral_obc: int, pdefweno: int,
                               stream: Any | None = None) -> None:
    """The final-stage moisture chain on a stretched column
    (launch_cuda_gm1_child_stretched_pdef_moisture,
    src/cm1core/cuda_gm1_child_stretched_scalar.py:851): the terrain branch's
    rdsf(k), or the flat column's rdz*mh(k) with its own base state."""
    if not isinstance(column, StretchedColumn):
        raise TypeError("column must be a StretchedColumn")
    if column.flat:
        prof = column.mh
        if not isinstance(prof, torch.Tensor) or tuple(prof.shape) != (nk + 2,):
            raise ValueError(f"mh must be a ({nk + 2},) tensor")
        col = _VerticalColumn(1, None, _f32(prof, "mh"), float(column.rdz))
    else:
        prof = column.rdsf
        if not isinstance(prof, torch.Tensor) or tuple(prof.shape) != (nk + 3,):
            raise ValueError(f"rdsf must be a ({nk + 3},) tensor")
        col = _VerticalColumn(0, _f32(prof, "rdsf"), None, 0.0)
    s = _Chain(**{n: _f32(a[n], n) for n in CHAIN_NAMES})
    _native.check(_lib().gm1b_pdef_moisture_chain_column(ni, nj, nk, ctypes.byref(s), dttmp, dx, dy, weps, lateral_obc,
                                                         pdefweno, ctypes.byref(col), _st(stream, a["rru"].device)),
                  "gm1b_pdef_moisture_chain_column")


def post_acoustic_flux_column(a: Mapping[str, torch.Tensor], column: Any, *, ni: int, nj: int, nk: int, dx: float,
                              dy: float, stream: Any | None = None) -> None:
    """getdiv/getdivx on a stretched column (launch_cuda_gm1_child_stretched_post_acoustic,
    src/cm1core/cuda_gm1_child_stretched_moist.py:286): ``column`` is a
    gm1_b200.momentum.StretchedMomentumColumn (terrain branch or flat)."""
    from .momentum import StretchedMomentumColumn, _Column  # noqa: PLC0415

    if not isinstance(column, StretchedMomentumColumn):
        raise TypeError("column must be a StretchedMomentumColumn")
    ptr = {n: (_f32(getattr(column, n), n) if getattr(column, n) is not None else None)
           for n in ("rho0_padded", "sigma", "sigmaf", "rds", "rdsf", "mh")}
    col = _Column(1 if column.flat else 0, ptr["rho0_padded"], ptr["sigma"], ptr["sigmaf"], ptr["rds"], ptr["rdsf"],
                  float(column.ztop), ptr["mh"], None, None, float(column.rdz))
    s = _Post(**{n: _f32(a[n], n) for n in POST_NAMES})
    _native.check(_lib().gm1b_post_acoustic_flux_column(ni, nj, nk, ctypes.byref(s), dx, dy, ctypes.byref(col),
                                                        _st(stream, a["rru"].device)), "gm1b_post_acoustic_flux_column")


def moist_buoyancy_flat(dum8, c1, c2, wten, *, ni: int, nj: int, nk: int, stream: Any | None = None) -> None:
    """The flat column's buoyancy, into wten only (launch_cuda_gm1_flat_stretched_buoyancy,
    src/cm1core/cuda_gm1_child_stretched_moist.py:240)."""
    ptrs = [_f32(t, n) for t, n in zip((dum8, c1, c2, wten), ("dum8", "c1", "c2", "wten"))]
    _native.check(_lib().gm1b_moist_buoyancy_flat(ni, nj, nk, *ptrs, _st(stream, dum8.device)),
                  "gm1b_moist_buoyancy_flat")


def held_compose(a: Mapping[str, torch.Tensor], *, ni: int, nj: int, nk: int, dt: float,
                 stream: Any | None = None) -> None:
    s = _Held(**{n: _f32(a[n], n) for n in HELD_NAMES})
    _native.check(_lib().gm1b_held_compose(ni, nj, nk, ctypes.byref(s), dt, _st(stream, a["rho"].device)),
                  "gm1b_held_compose")


def solve3_density(rho, c1, c2, rr, rf, *, ni: int, nj: int, nk: int, stream: Any | None = None) -> None:
    ptrs = [_f32(t, n) for t, n in zip((rho, c1, c2, rr, rf), ("rho", "c1", "c2", "rr", "rf"))]
    _native.check(_lib().gm1b_solve3_density(ni, nj, nk, *ptrs, _st(stream, rho.device)), "gm1b_solve3_density")


def pack_scalar(scalar, padded, *, ni: int, nj: int, nk: int, stream: Any | None = None) -> None:
    _native.check(_lib().gm1b_pack_scalar(ni, nj, nk, _f32(scalar, "scalar"), _f32(padded, "padded"),
                                          _st(stream, scalar.device)), "gm1b_pack_scalar")



def bcwsfc(u3d, v3d, w3d, gz, dzdx, dzdy, *, ni: int, nj: int, nk: int, stream: Any | None = None) -> None:
    ptrs = [_f32(t, n) for t, n in zip((u3d, v3d, w3d, gz, dzdx, dzdy), ("u3d", "v3d", "w3d", "gz", "dzdx", "dzdy"))]
    _native.check(_lib().gm1b_bcwsfc(ni, nj, nk, *ptrs, _st(stream, u3d.device)), "gm1b_bcwsfc")


def w_level1_fill(w3d, *, ni: int, nj: int, nk: int, stream: Any | None = None) -> None:
    _native.check(_lib().gm1b_w_level1_fill(ni, nj, nk, _f32(w3d, "w3d"), _st(stream, w3d.device)),
                  "gm1b_w_level1_fill")
