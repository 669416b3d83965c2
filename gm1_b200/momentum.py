"""Terrain/open fifth-order momentum advection on B200.

Drop-in mirror of the reference operator API (torch CUDA tensors in place of
CuPy arrays; the same names, keywords, contracts and errors):

  MomentumAdvection5Selection, validate_...       src/cm1core/cuda_momentum_advection5.py:82-233
  momentum_lateral_sides, momentum_open_boundary_code,
  momentum_advection5_counts, momentum_boundary_faces   :103-165
  launch_cuda_terrain_open_momentum_advection5    :1173-1330

The mass fluxes and divx are one library call (gm1b_momentum_mass_flux5) and
advu / advv / advw another (gm1b_momentum_transport5); both hooks of the
reference run between the two on the same stream.  rrw_boundary_hook runs
after divx here rather than before it: divx reads rrw in the physical columns
only and the hook fills lateral halo columns only, so the words are the same.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Any, Callable, Mapping

import torch

from . import _native

NGXY = 3
MOMENTUM_ALL_OPEN_SIDES = (2, 2, 2, 2)
_STRUCT = ("u3d", "uten", "rru", "v3d", "vten", "rrv", "w3d", "wten", "rrw", "uh", "vh", "rho0_3d", "rf0", "rrf0",
           "c2", "gz", "gzu", "gzv", "rgzu", "rgzv", "dzdx", "dzdy", "divx")
_STATE = ("u3d", "uten", "rru", "v3d", "vten", "rrv", "w3d", "wten", "rrw", "uh", "vh")
_WRITABLE = ("uten", "vten", "wten", "rru", "rrv", "rrw")
_METRICS = ("rho0_3d", "rf0", "rr0", "rrf0", "c1", "c2", "gz", "gzu", "gzv", "rgzu", "rgzv", "dzdx", "dzdy")
_RRW_HOOK_SCHEMA = "gm1.cuda-bcw-rrw-open-flag0/v1"


@dataclass(frozen=True, slots=True)
class MomentumAdvection5Selection:
    hadvordrv: int = 5
    vadvordrv: int = 5
    advwenov: int = 0
    axisymmetric: int = 0
    terrain: bool = True
    idiff: int = 0
    immersed_boundary: bool = False
    uniform_horizontal_grid: bool = True
    uniform_vertical_sigma: bool = True
    lateral_boundaries: tuple[int, int, int, int] = (2, 2, 2, 2)


DEFAULT_MOMENTUM_ADVECTION5_SELECTION = MomentumAdvection5Selection()


def momentum_lateral_sides(lateral_sides: Any) -> tuple[int, int, int, int]:
    """CM1's (wbc, ebc, sbc, nbc), each 1 (periodic), 2 (open), 3 or 4
    (walls); one-sided periodic directions are refused as param.F does."""
    sides = tuple(lateral_sides)
    if len(sides) != 4 or any(isinstance(v, bool) or not isinstance(v, int) or v not in (1, 2, 3, 4) for v in sides):
        raise ValueError("lateral_sides must be CM1's (wbc, ebc, sbc, nbc), each 1, 2, 3 or 4")
    if (sides[0] == 1) != (sides[1] == 1) or (sides[2] == 1) != (sides[3] == 1):
        raise ValueError(f"lateral_sides {sides}: param.F:2562-2588 stops CM1 when only one side of a direction "
                         "is periodic")
    return sides  # type: ignore[return-value]


def momentum_open_boundary_code(lateral_sides: Any) -> int:
    """The packed obc word: wbc | ebc << 4 | sbc << 8 | nbc << 12."""
    w, e, s, n = momentum_lateral_sides(lateral_sides)
    return w | (e << 4) | (s << 8) | (n << 12)


def momentum_advection5_counts(ni: int, nj: int, nk: int,
                               lateral_sides: Any = MOMENTUM_ALL_OPEN_SIDES) -> tuple[int, int, int]:
    """Words advu, advv and advw update: faces i1..i2, rows j1..j2, every
    interior w level."""
    w, e, s, n = momentum_lateral_sides(lateral_sides)
    faces = ni - 1 + int(w == 1) + int(e == 1)
    rows = nj - 1 + int(s == 1) + int(n == 1)
    return nk * nj * faces, nk * rows * ni, (nk - 1) * nj * ni


def momentum_boundary_faces(lateral_sides: Any) -> dict[str, Any]:
    w, e, s, n = momentum_lateral_sides(lateral_sides)
    return {
        "advu_faces_one_based": [1 if w == 1 else 2, "ni+1" if e == 1 else "ni"],
        "advv_rows_one_based": [1 if s == 1 else 2, "nj+1" if n == 1 else "nj"],
        "inflow_edits_on": [name for name, side in zip(("west", "east", "south", "north"), (w, e, s, n))
                            if side == 2],
    }


def validate_momentum_advection5_selection(selection: MomentumAdvection5Selection) -> None:
    if not isinstance(selection, MomentumAdvection5Selection):
        raise TypeError("selection must be MomentumAdvection5Selection")
    expected = DEFAULT_MOMENTUM_ADVECTION5_SELECTION
    if selection != expected:
        for name in ("hadvordrv", "vadvordrv", "advwenov", "axisymmetric", "terrain", "idiff", "immersed_boundary",
                     "uniform_horizontal_grid", "uniform_vertical_sigma", "lateral_boundaries"):
            if getattr(selection, name) != getattr(expected, name):
                raise ValueError(f"unsupported momentum-advection selection {name}={getattr(selection, name)!r}; "
                                 f"required {getattr(expected, name)!r}")


def momentum_advection5_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    ng = NGXY
    u, v, w = (nk + 2, nj + 2 * ng, ni + 1 + 2 * ng), (nk + 2, nj + 1 + 2 * ng, ni + 2 * ng), \
        (nk + 3, nj + 2 * ng, ni + 2 * ng)
    mass, face = (nk, nj, ni), (nk + 1, nj, ni)
    return {"u3d": u, "uten": u, "rru": u, "v3d": v, "vten": v, "rrv": v, "w3d": w, "wten": w, "rrw": w,
            "uh": (ni + 2 * ng,), "vh": (nj + 2 * ng,), "rho0_3d": mass, "rf0": face, "rr0": mass, "rrf0": face,
            "c1": face, "c2": face, "gz": (nj, ni), "gzu": (nj, ni + 1), "gzv": (nj + 1, ni), "rgzu": (nj, ni + 1),
            "rgzv": (nj + 1, ni), "dzdx": (nj, ni), "dzdy": (nj, ni), "divx": mass}


class _Arrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in _STRUCT]


@dataclass(slots=True)
class CudaMomentumAdvection5Launch:
    divx: torch.Tensor
    ready_event: torch.cuda.Event
    receipt: dict[str, Any]


class _Column(ctypes.Structure):
    _fields_ = [("flat", ctypes.c_int32), ("rho0_padded", ctypes.c_void_p), ("sigma", ctypes.c_void_p),
                ("sigmaf", ctypes.c_void_p), ("rds", ctypes.c_void_p), ("rdsf", ctypes.c_void_p),
                ("ztop", ctypes.c_float), ("mh", ctypes.c_void_p), ("mf", ctypes.c_void_p), ("rr0", ctypes.c_void_p),
                ("rdz", ctypes.c_float)]


@dataclass(frozen=True)
class StretchedMomentumColumn:
    """The vertical column of the stretched momentum operator (the profiles
    the reference binds from its Gm1ChildStretchedMetrics): ``rho0_padded`` the
    (nk+2, nj+6, ni+6) base density; terrain branch (``flat=False``) with
    ``sigma`` (nk+2), ``sigmaf`` (nk+3), ``rds`` (nk+2), ``rdsf`` (nk+3) and the
    physical top ``ztop``; flat column (``flat=True``) with ``mh`` (nk+2),
    ``mf`` (nk+3), ``rr0`` (nk, nj, ni) and ``rdz``."""

    flat: bool
    rho0_padded: Any
    sigma: Any = None
    sigmaf: Any = None
    rds: Any = None
    rdsf: Any = None
    ztop: float = 0.0
    mh: Any = None
    mf: Any = None
    rr0: Any = None
    rdz: float = 0.0


def _lib():
    lib = _native.lib()
    if not getattr(lib, "_mom5_bound", False):
        i32, u32, f32, vp = ctypes.c_int32, ctypes.c_uint32, ctypes.c_float, ctypes.c_void_p
        for fn in (lib.gm1b_momentum_advection5, lib.gm1b_momentum_mass_flux5, lib.gm1b_momentum_transport5):
            fn.argtypes = [i32, i32, i32, ctypes.POINTER(_Arrays), u32, f32, f32, f32, vp]
            fn.restype = i32
        for fn in (lib.gm1b_momentum_advection5_column, lib.gm1b_momentum_mass_flux5_column,
                   lib.gm1b_momentum_transport5_column):
            fn.argtypes = [i32, i32, i32, ctypes.POINTER(_Arrays), u32, f32, f32, ctypes.POINTER(_Column), vp]
            fn.restype = i32
        lib._mom5_bound = True
    return lib


def _positive_int(name: str, value: object, minimum: int) -> int:
    if isinstance(value, bool) or not isinstance(value, int) or value < minimum:
        raise ValueError(f"{name} must be an integer >= {minimum}")
    return value


def _spacing(name: str, value: object) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise TypeError(f"{name} must be numeric")
    x = float(value)
    if not math.isfinite(x) or x <= 0.0:
        raise ValueError(f"{name} must be finite and > 0")
    return x


def _require_cuda(value: Any, name: str, shape: tuple[int, ...]) -> torch.Tensor:
    if not isinstance(value, torch.Tensor) or not value.is_cuda or value.dtype != torch.float32:
        raise TypeError(f"{name} must be a float32 CUDA tensor")
    if tuple(value.shape) != shape or not value.is_contiguous():
        raise ValueError(f"{name} must have C-order shape {shape}")
    return value


def _spans(t: torch.Tensor) -> tuple[int, int]:
    return t.data_ptr(), t.data_ptr() + t.numel() * 4


def launch_cuda_terrain_open_momentum_advection5(
        arrays: Mapping[str, Any], metrics: Mapping[str, Any], *, ni: int, nj: int, nk: int, nrk: int, dx: float,
        dy: float, dz: float, divx: Any | None = None,
        selection: MomentumAdvection5Selection = DEFAULT_MOMENTUM_ADVECTION5_SELECTION, stream: Any | None = None,
        rrw_boundary_hook: Any | None = None,
        post_divergence_hook: Callable[..., Mapping[str, object]] | None = None,
        lateral_sides: tuple[int, int, int, int] = MOMENTUM_ALL_OPEN_SIDES) -> CudaMomentumAdvection5Launch:
    """Enqueue rru/rrv/rrw, divx and the advu/advv/advw increments of
    uten/vten/wten for the lateral family ``lateral_sides``; the hooks run
    on ``stream`` between divx and advu (solve2.F:631-720's seam)."""
    validate_momentum_advection5_selection(selection)
    lateral_sides = momentum_lateral_sides(lateral_sides)
    obc = momentum_open_boundary_code(lateral_sides)
    if rrw_boundary_hook is not None and not callable(rrw_boundary_hook):
        raise TypeError("rrw_boundary_hook must be callable or None")
    if post_divergence_hook is not None and not callable(post_divergence_hook):
        raise TypeError("post_divergence_hook must be callable or None")
    ni = _positive_int("ni", ni, 7)
    nj = _positive_int("nj", nj, 7)
    nk = _positive_int("nk", nk, 8)
    if isinstance(nrk, bool) or not isinstance(nrk, int) or nrk not in (1, 2, 3):
        raise ValueError("nrk must be an integer in 1..3")
    dx, dy, dz = (_spacing(n, v) for n, v in (("dx", dx), ("dy", dy), ("dz", dz)))
    shapes = momentum_advection5_shapes(ni, nj, nk)
    a = {n: _require_cuda(arrays[n], n, shapes[n]) for n in _STATE}
    m = {n: _require_cuda(metrics[n], n, shapes[n]) for n in _METRICS}
    device = a["u3d"].device
    if divx is None:
        divx = torch.empty((nk, nj, ni), dtype=torch.float32, device=device)
    else:
        divx = _require_cuda(divx, "divx", (nk, nj, ni))
    mutable = [a[n] for n in _WRITABLE] + [divx]
    others = [a[n] for n in _STATE if n not in _WRITABLE] + list(m.values())
    for i, t in enumerate(mutable):
        lo, hi = _spans(t)
        for o in mutable[i + 1:] + others:
            olo, ohi = _spans(o)
            if lo < ohi and olo < hi:
                raise ValueError("momentum-advection mutable arrays and metrics must not alias")
    lib = _lib()
    st = torch.cuda.current_stream(device) if stream is None else stream
    s = _Arrays(**{n: (divx if n == "divx" else a[n] if n in a else m[n]).data_ptr() for n in _STRUCT})
    args = (ni, nj, nk, ctypes.byref(s), obc, dx, dy, dz, ctypes.c_void_p(st.cuda_stream))
    rrw_receipt = post_receipt = None
    with torch.cuda.device(device), torch.cuda.stream(st):
        if rrw_boundary_hook is None and post_divergence_hook is None:
            _native.check(lib.gm1b_momentum_advection5(*args), "gm1b_momentum_advection5")
        else:
            _native.check(lib.gm1b_momentum_mass_flux5(*args), "gm1b_momentum_mass_flux5")
            if rrw_boundary_hook is not None:
                rrw_receipt = rrw_boundary_hook(a["rrw"], stream=st, ni=ni, nj=nj, nk=nk)
                if not isinstance(rrw_receipt, Mapping) or rrw_receipt.get("performed") is not True \
                        or rrw_receipt.get("flag") != 0 or rrw_receipt.get("vertical_rigid_faces_written") is not False \
                        or rrw_receipt.get("stream_pointer") != int(st.cuda_stream) \
                        or rrw_receipt.get("schema") != _RRW_HOOK_SCHEMA \
                        or list(rrw_receipt.get("directions") or ()) != ["west", "east", "south", "north"]:
                    raise ValueError("bcw(rrw,0) hook did not confirm source-ordered same-stream lateral-only filling")
            if post_divergence_hook is not None:
                post_receipt = post_divergence_hook(a, stream=st, ni=ni, nj=nj, nk=nk, nrk=nrk, ng=NGXY)
                if not isinstance(post_receipt, Mapping):
                    raise TypeError("post_divergence_hook must return a receipt mapping")
            _native.check(lib.gm1b_momentum_transport5(*args), "gm1b_momentum_transport5")
        ev = torch.cuda.Event()
        ev.record(st)
    receipt: dict[str, Any] = {
        "selection": {"hadvordrv": 5, "vadvordrv": 5, "advwenov": 0, "axisymmetric": 0, "terrain": True, "idiff": 0,
                      "immersed_boundary": False, "uniform_horizontal_grid": True, "uniform_vertical_sigma": True,
                      "lateral_boundaries": list(lateral_sides), "nrk": nrk},
        "boundary_faces": momentum_boundary_faces(lateral_sides),
        "domain": {"ni": ni, "nj": nj, "nk": nk},
        "launches": 3,
    }
    if rrw_receipt is not None:
        receipt["rrw_open_boundary"] = dict(rrw_receipt)
    if post_receipt is not None:
        receipt["post_divergence"] = dict(post_receipt)
    return CudaMomentumAdvection5Launch(divx, ev, receipt)


def launch_cuda_gm1_child_stretched_momentum5(
        arrays: Mapping[str, Any], metrics: Mapping[str, Any], vertical: StretchedMomentumColumn, *, ni: int, nj: int,
        nk: int, nrk: int, dx: float, dy: float, divx: Any | None = None, stream: Any | None = None,
        rrw_boundary_hook: Any | None = None,
        lateral_sides: tuple[int, int, int, int] = MOMENTUM_ALL_OPEN_SIDES) -> CudaMomentumAdvection5Launch:
    """The momentum advection on a stretched column
    (launch_cuda_gm1_child_stretched_momentum5,
    src/cm1core/cuda_gm1_child_stretched_momentum.py:540): terrain branch
    (rdsf / rds / sigma / sigmaf, the physical top) or flat column
    (rdz*mh / rdz*mf and the column's base state).  ``rrw_boundary_hook``
    runs between the mass fluxes and the transport (a terrain-branch
    bcw(rrw,0); a flat column takes none)."""
    if not isinstance(vertical, StretchedMomentumColumn):
        raise TypeError("vertical must be a StretchedMomentumColumn")
    if vertical.flat and rrw_boundary_hook is not None:
        raise ValueError("solve2.F:575's bcw(rrw,0) is a terrain statement: a flat column takes no rrw hook")
    lateral_sides = momentum_lateral_sides(lateral_sides)
    obc = momentum_open_boundary_code(lateral_sides)
    ni = _positive_int("ni", ni, 7)
    nj = _positive_int("nj", nj, 7)
    nk = _positive_int("nk", nk, 8)
    if isinstance(nrk, bool) or not isinstance(nrk, int) or nrk not in (1, 2, 3):
        raise ValueError("nrk must be an integer in 1..3")
    dx, dy = (_spacing(n, v) for n, v in (("dx", dx), ("dy", dy)))
    shapes = momentum_advection5_shapes(ni, nj, nk)
    a = {n: _require_cuda(arrays[n], n, shapes[n]) for n in _STATE}
    m = {n: _require_cuda(metrics[n], n, shapes[n]) for n in _METRICS}
    device = a["u3d"].device
    divx = torch.empty((nk, nj, ni), dtype=torch.float32, device=device) if divx is None else \
        _require_cuda(divx, "divx", (nk, nj, ni))
    rho0p = _require_cuda(vertical.rho0_padded, "rho0_padded", (nk + 2, nj + 6, ni + 6))
    prof = {}
    if vertical.flat:
        for n, shape in (("mh", (nk + 2,)), ("mf", (nk + 3,)), ("rr0", (nk, nj, ni))):
            prof[n] = _require_cuda(getattr(vertical, n), n, shape)
        rdz = float(vertical.rdz)
        if not (math.isfinite(rdz) and rdz > 0.0):
            raise ValueError("a flat column needs rdz > 0")
        col = _Column(1, rho0p.data_ptr(), None, None, None, None, 0.0, prof["mh"].data_ptr(), prof["mf"].data_ptr(),
                      prof["rr0"].data_ptr(), rdz)
    else:
        for n, shape in (("sigma", (nk + 2,)), ("sigmaf", (nk + 3,)), ("rds", (nk + 2,)), ("rdsf", (nk + 3,))):
            prof[n] = _require_cuda(getattr(vertical, n), n, shape)
        ztop = float(vertical.ztop)
        if not (math.isfinite(ztop) and ztop > 0.0):
            raise ValueError("a terrain column needs its physical top ztop > 0")
        col = _Column(0, rho0p.data_ptr(), prof["sigma"].data_ptr(), prof["sigmaf"].data_ptr(),
                      prof["rds"].data_ptr(), prof["rdsf"].data_ptr(), ztop, None, None, None, 0.0)
    mutable = [a[n] for n in _WRITABLE] + [divx]
    others = [a[n] for n in _STATE if n not in _WRITABLE] + list(m.values()) + [rho0p] + list(prof.values())
    for i, t in enumerate(mutable):
        lo, hi = _spans(t)
        for o in mutable[i + 1:] + others:
            olo, ohi = _spans(o)
            if lo < ohi and olo < hi:
                raise ValueError("stretched momentum mutable arrays, metrics and profiles must not alias")
    lib = _lib()
    st = torch.cuda.current_stream(device) if stream is None else stream
    s = _Arrays(**{n: (divx if n == "divx" else a[n] if n in a else m[n]).data_ptr() for n in _STRUCT})
    args = (ni, nj, nk, ctypes.byref(s), obc, dx, dy, ctypes.byref(col), ctypes.c_void_p(st.cuda_stream))
    rrw_receipt = None
    with torch.cuda.device(device), torch.cuda.stream(st):
        if rrw_boundary_hook is None:
            _native.check(lib.gm1b_momentum_advection5_column(*args), "gm1b_momentum_advection5_column")
        else:
            _native.check(lib.gm1b_momentum_mass_flux5_column(*args), "gm1b_momentum_mass_flux5_column")
            rrw_receipt = rrw_boundary_hook(a["rrw"], stream=st, ni=ni, nj=nj, nk=nk)
            _native.check(lib.gm1b_momentum_transport5_column(*args), "gm1b_momentum_transport5_column")
        ev = torch.cuda.Event()
        ev.record(st)
    receipt: dict[str, Any] = {"terrain": not vertical.flat, "stretch_z": 1, "nrk": nrk,
                               "lateral_boundaries": list(lateral_sides), "domain": {"ni": ni, "nj": nj, "nk": nk},
                               "launches": 3}
    if rrw_receipt is not None:
        receipt["rrw_open_boundary"] = dict(rrw_receipt)
    return CudaMomentumAdvection5Launch(divx, ev, receipt)
