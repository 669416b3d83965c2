"""Fifth-order / WENO5 scalar advection and the terrain mass flux on the
padded (ng = 3) lane, on B200.

Drop-in mirrors of the reference operator API (torch CUDA tensors in place of
CuPy arrays; same dictionary keys, shapes, keywords and refusals):

  Advection5Selection, scalar_advection_uses_weno
                                  src/cm1core/cuda_advection5.py:60-147
  launch_cuda_terrain_mass_flux5  src/cm1core/cuda_advection5.py:849
  launch_cuda_scalar_advection5   src/cm1core/cuda_advection5.py:948

The CUDA kernels (libgm1b.so, advection5.cu) are bit-identical to the
reference's CPU twins.  The scalar pass is fused: the face fluxes never go
through HBM unless ``write_fluxes`` asks for the reference's flux outputs.
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

CM1_OPEN_NGXY = 3
CM1_NRKMAX = 3
CM1_WENO_SIFORM = 2


@dataclass(frozen=True, slots=True)
class Advection5Selection:
    scalar_horizontal_order: int = 5
    scalar_vertical_order: int = 5
    scalar_weno: int = 2
    velocity_horizontal_order: int = 5
    velocity_vertical_order: int = 5
    velocity_weno: int = 0
    weno_order: int = 5
    weno_siform: int = CM1_WENO_SIFORM
    terrain: bool = True
    axisymmetric: int = 0
    mpi: bool = False
    positive_definite: bool = False


DEFAULT_ADVECTION5_SELECTION = Advection5Selection()
_EXPECTED = {
    "dynamics.scalar_horizontal_order": ("scalar_horizontal_order", 5),
    "dynamics.scalar_vertical_order": ("scalar_vertical_order", 5),
    "dynamics.scalar_weno": ("scalar_weno", 2),
    "dynamics.velocity_horizontal_order": ("velocity_horizontal_order", 5),
    "dynamics.velocity_vertical_order": ("velocity_vertical_order", 5),
    "dynamics.velocity_weno": ("velocity_weno", 0),
    "dynamics.weno_order": ("weno_order", 5),
    "dynamics.weno_siform": ("weno_siform", 2),
    "grid.terrain": ("terrain", True),
    "grid.axisymmetric": ("axisymmetric", 0),
    "runtime.mpi": ("mpi", False),
    "advection.positive_definite": ("positive_definite", False),
}


def validate_advection5_selection(selection: Advection5Selection) -> None:
    """Refuse every branch other than the admitted fifth-order/WENO-Z one
    (src/cm1core/cuda_advection5.py:93-126)."""
    if not isinstance(selection, Advection5Selection):
        raise TypeError("selection must be an Advection5Selection")
    for option, (attribute, expected) in _EXPECTED.items():
        value = getattr(selection, attribute)
        if type(value) is not type(expected) or value != expected:
            refuse(
                code="CM1-ADVECTION5-UNSUPPORTED",
                gate="dry-dynamics",
                option=option,
                value=value,
                reason="only the fifth-order terrain scalar branch with final-stage WENO-Z is built; "
                "another value selects a different stencil, cadence or geometry",
                remedy="use the fifth-order/WENO-Z profile",
            )


def scalar_advection_uses_weno(
    nrk: int, *, nrkmax: int = CM1_NRKMAX, wflag: bool = True,
    selection: Advection5Selection = DEFAULT_ADVECTION5_SELECTION,
) -> bool:
    """WENO iff wflag and nrk == nrkmax (src/cm1core/cuda_advection5.py:129-147)."""
    validate_advection5_selection(selection)
    if isinstance(nrk, bool) or not isinstance(nrk, int):
        raise TypeError("nrk must be an integer")
    if isinstance(nrkmax, bool) or not isinstance(nrkmax, int):
        raise TypeError("nrkmax must be an integer")
    if nrkmax != CM1_NRKMAX or nrk < 1 or nrk > nrkmax:
        raise ValueError("the sealed low-storage schedule requires nrkmax=3 and nrk=1..3")
    if not isinstance(wflag, bool):
        raise TypeError("wflag must be boolean")
    return bool(wflag and selection.scalar_weno == 2 and nrk == nrkmax)


def scalar_open_boundary_code(lateral_sides: tuple[int, int, int, int] | None) -> int:
    """Pack CM1's (wbc, ebc, sbc, nbc) as wbc | ebc<<4 | sbc<<8 | nbc<<12;
    None is a tile-local launch (0)."""
    if lateral_sides is None:
        return 0
    sides = tuple(lateral_sides)
    if len(sides) != 4 or any(isinstance(v, bool) or not isinstance(v, int) or v not in (1, 2, 3, 4) for v in sides):
        raise ValueError("lateral_sides must be CM1's (wbc, ebc, sbc, nbc), each 1, 2, 3 or 4")
    return sides[0] | (sides[1] << 4) | (sides[2] << 8) | (sides[3] << 12)


def padded_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    ng = CM1_OPEN_NGXY
    return {
        "scalar": (nk + 2, nj + 2 * ng, ni + 2 * ng),
        "u": (nk + 2, nj + 2 * ng, ni + 1 + 2 * ng),
        "v": (nk + 2, nj + 1 + 2 * ng, ni + 2 * ng),
        "w": (nk + 3, nj + 2 * ng, ni + 2 * ng),
        "cell": (nk, nj, ni),
        "face": (nk + 1, nj, ni),
    }


def _validated_grid(ni: int, nj: int, nk: int) -> None:
    for name, value in (("ni", ni), ("nj", nj), ("nk", nk)):
        if isinstance(value, bool) or not isinstance(value, int) or value < 8:
            raise ValueError(f"{name} must be an integer >= 8")


def _validated_spacing(name: str, value: float) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise TypeError(f"{name} must be numeric")
    result = float(value)
    if not math.isfinite(result) or result <= 0.0:
        raise ValueError(f"{name} must be finite and > 0")
    return result


def _require(value: Any, name: str, shape: tuple[int, ...]) -> torch.Tensor:
    if not isinstance(value, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if not value.is_cuda or value.dtype != torch.float32 or tuple(value.shape) != shape or not value.is_contiguous():
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor of shape {shape}")
    return value


def _no_alias(tensors: list[torch.Tensor], what: str) -> None:
    ptrs = [t.data_ptr() for t in tensors]
    if len(ptrs) != len(set(ptrs)):
        raise ValueError(f"{what} must not alias")


class _MassFluxArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("u3d", "v3d", "w3d", "rru", "rrv", "rrw", "rho0_3d", "rf0", "rgzu",
                                               "rgzv", "dzdx", "dzdy", "gz", "divx")]


class _ScalarAdvArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("scalar", "rru", "rrv", "rrw", "c1", "c2", "rr0", "gz", "divx",
                                               "tendency", "flux_x", "flux_y", "flux_z")]


class _VerticalColumn(ctypes.Structure):
    _fields_ = [("flat", ctypes.c_int32), ("rdsf", ctypes.c_void_p), ("mh", ctypes.c_void_p), ("rdz", ctypes.c_float)]


@dataclass(frozen=True)
class StretchedColumn:
    """The vertical column a stretched-grid operator reads (the profiles the
    reference binds from its Gm1ChildStretchedMetrics): ``flat=False`` is
    CM1's terrain branch with ``rdsf`` (nk+3 words, CM1-indexed: 1/(sigmaf(k+1)
    - sigmaf(k)) at k = 1..nk); ``flat=True`` the flat column with ``mh``
    (nk+2 words) and ``rdz`` = 1/dz of the metric reference."""

    flat: bool
    rdsf: Any = None
    mh: Any = None
    rdz: float = 0.0


def _bind() -> ctypes.CDLL:
    lib = _native.lib()
    if not getattr(lib, "_adv_bound", False):
        i32, f32, vp = ctypes.c_int32, ctypes.c_float, ctypes.c_void_p
        lib.gm1b_terrain_mass_flux5.argtypes = [i32, i32, i32, ctypes.POINTER(_MassFluxArrays), f32, f32, f32, vp]
        lib.gm1b_terrain_mass_flux5.restype = i32
        lib.gm1b_scalar_advection5_column.argtypes = [i32, i32, i32, ctypes.POINTER(_ScalarAdvArrays), i32, i32, f32,
                                                      f32, ctypes.c_double, ctypes.c_uint32, i32,
                                                      ctypes.POINTER(_VerticalColumn), ctypes.c_void_p]
        lib.gm1b_scalar_advection5_column.restype = i32
        lib.gm1b_scalar_advection5.argtypes = [i32, i32, i32, ctypes.POINTER(_ScalarAdvArrays), i32, i32, f32, f32,
                                               f32, ctypes.c_double, ctypes.c_uint32, i32, vp]
        lib.gm1b_scalar_advection5.restype = i32
        lib._adv_bound = True
    return lib


def launch_cuda_terrain_mass_flux5(
    arrays: Mapping[str, Any], metrics: Mapping[str, Any], divx: Any, *, ni: int, nj: int, nk: int,
    dx: float, dy: float, dz: float, selection: Advection5Selection = DEFAULT_ADVECTION5_SELECTION,
    stream: Any | None = None,
) -> CudaLaunch:
    """Enqueue the terrain mass flux (interior faces) and interior divergence."""
    validate_advection5_selection(selection)
    _validated_grid(ni, nj, nk)
    dx, dy, dz = (_validated_spacing(n, v) for n, v in (("dx", dx), ("dy", dy), ("dz", dz)))
    sh = padded_shapes(ni, nj, nk)
    a = {
        "u3d": _require(arrays["u3d"], "u3d", sh["u"]), "v3d": _require(arrays["v3d"], "v3d", sh["v"]),
        "w3d": _require(arrays["w3d"], "w3d", sh["w"]), "rru": _require(arrays["rru"], "rru", sh["u"]),
        "rrv": _require(arrays["rrv"], "rrv", sh["v"]), "rrw": _require(arrays["rrw"], "rrw", sh["w"]),
        "rho0_3d": _require(metrics["rho0_3d"], "rho0_3d", sh["cell"]),
        "rf0": _require(metrics["rf0"], "rf0", sh["face"]),
        "rgzu": _require(metrics["rgzu"], "rgzu", (nj, ni + 1)), "rgzv": _require(metrics["rgzv"], "rgzv", (nj + 1, ni)),
        "dzdx": _require(metrics["dzdx"], "dzdx", (nj, ni)), "dzdy": _require(metrics["dzdy"], "dzdy", (nj, ni)),
        "gz": _require(metrics["gz"], "gz", (nj, ni)), "divx": _require(divx, "divx", sh["cell"]),
    }
    _no_alias(list(a.values()), "terrain mass-flux inputs and outputs")
    s = _MassFluxArrays(**{n: t.data_ptr() for n, t in a.items()})
    device = a["u3d"].device
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        _native.check(_bind().gm1b_terrain_mass_flux5(ni, nj, nk, ctypes.byref(s), dx, dy, dz,
                                                      ctypes.c_void_p(st.cuda_stream)), "gm1b_terrain_mass_flux5")
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {"operation": "terrain-mass-flux-and-divergence", "domain": {"ni": ni, "nj": nj, "nk": nk}})


def launch_cuda_scalar_advection5(
    scalar: Any, arrays: Mapping[str, Any], metrics: Mapping[str, Any], divx: Any, tendency: Any,
    fluxes: Mapping[str, Any] | None, *, ni: int, nj: int, nk: int, nrk: int, dx: float, dy: float, dz: float,
    weps: float, wflag: bool = True, selection: Advection5Selection = DEFAULT_ADVECTION5_SELECTION,
    stream: Any | None = None, lateral_sides: tuple[int, int, int, int] | None = None,
    write_fluxes: bool = True, levels_per_chunk: int | None = None,
) -> CudaLaunch:
    """Enqueue one scalar's fifth-order/WENO5 tendency for RK stage ``nrk``.

    ``lateral_sides`` is CM1's (wbc, ebc, sbc, nbc) of a whole-domain launch;
    None is a tile-local launch whose outer three cells are not written.
    ``write_fluxes`` also stores the face fluxes into ``fluxes`` x/y/z as the
    reference does; False skips those HBM writes (``fluxes`` may be None)."""
    use_weno = scalar_advection_uses_weno(nrk, wflag=wflag, selection=selection)
    _validated_grid(ni, nj, nk)
    dx, dy, dz = (_validated_spacing(n, v) for n, v in (("dx", dx), ("dy", dy), ("dz", dz)))
    if isinstance(weps, bool) or not isinstance(weps, (int, float)):
        raise TypeError("weps must be numeric")
    weps = float(weps)
    if not math.isfinite(weps) or weps <= 0.0:
        raise ValueError("weps must be finite and > 0")
    obc = scalar_open_boundary_code(lateral_sides)
    sh = padded_shapes(ni, nj, nk)
    a = {
        "scalar": _require(scalar, "scalar", sh["scalar"]),
        "rru": _require(arrays["rru"], "rru", sh["u"]), "rrv": _require(arrays["rrv"], "rrv", sh["v"]),
        "rrw": _require(arrays["rrw"], "rrw", sh["w"]),
        "c1": _require(metrics["c1"], "c1", sh["face"]), "c2": _require(metrics["c2"], "c2", sh["face"]),
        "rr0": _require(metrics["rr0"], "rr0", sh["cell"]), "gz": _require(metrics["gz"], "gz", (nj, ni)),
        "divx": _require(divx, "divx", sh["cell"]), "tendency": _require(tendency, "tendency", sh["cell"]),
    }
    if write_fluxes:
        if fluxes is None:
            raise ValueError("write_fluxes requires the fluxes x/y/z arrays")
        a["flux_x"] = _require(fluxes["x"], "flux_x", sh["u"])
        a["flux_y"] = _require(fluxes["y"], "flux_y", sh["v"])
        a["flux_z"] = _require(fluxes["z"], "flux_z", sh["w"])
    _no_alias(list(a.values()), "scalar advection inputs, flux scratch, and tendency")
    s = _ScalarAdvArrays(**{n: t.data_ptr() for n, t in a.items()})
    device = a["scalar"].device
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        _native.check(_bind().gm1b_scalar_advection5(ni, nj, nk, ctypes.byref(s), nrk, 1 if wflag else 0, dx, dy, dz,
                                                     weps, obc, int(levels_per_chunk or 0),
                                                     ctypes.c_void_p(st.cuda_stream)), "gm1b_scalar_advection5")
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {"operation": "scalar-advection5", "nrk": nrk, "weno": use_weno, "lateral_obc": obc})


def launch_cuda_gm1_child_stretched_scalar_advection5(
    scalar: Any, arrays: Mapping[str, Any], metrics: Mapping[str, Any], divx: Any, tendency: Any,
    fluxes: Mapping[str, Any] | None, vertical: StretchedColumn, *, ni: int, nj: int, nk: int, nrk: int, dx: float,
    dy: float, weps: float, wflag: bool = True, stream: Any | None = None,
    lateral_sides: tuple[int, int, int, int] | None = None, write_fluxes: bool = True,
    levels_per_chunk: int | None = None,
) -> CudaLaunch:
    """The scalar tendency on a stretched column
    (launch_cuda_gm1_child_stretched_scalar_advection5,
    src/cm1core/cuda_gm1_child_stretched_scalar.py:666): the fluxes of
    launch_cuda_scalar_advection5, the vertical derivative with the column's
    own rdsf(k) (terrain branch) or rdz*mh(k) and rr0(k) (flat column)."""
    if not isinstance(vertical, StretchedColumn):
        raise TypeError("vertical must be a StretchedColumn")
    use_weno = scalar_advection_uses_weno(nrk, wflag=wflag)
    _validated_grid(ni, nj, nk)
    dx, dy = (_validated_spacing(n, v) for n, v in (("dx", dx), ("dy", dy)))
    if isinstance(weps, bool) or not isinstance(weps, (int, float)):
        raise TypeError("weps must be numeric")
    weps = float(weps)
    if not math.isfinite(weps) or weps <= 0.0:
        raise ValueError("weps must be finite and > 0")
    obc = scalar_open_boundary_code(lateral_sides)
    sh = padded_shapes(ni, nj, nk)
    a = {
        "scalar": _require(scalar, "scalar", sh["scalar"]),
        "rru": _require(arrays["rru"], "rru", sh["u"]), "rrv": _require(arrays["rrv"], "rrv", sh["v"]),
        "rrw": _require(arrays["rrw"], "rrw", sh["w"]),
        "c1": _require(metrics["c1"], "c1", sh["face"]), "c2": _require(metrics["c2"], "c2", sh["face"]),
        "rr0": _require(metrics["rr0"], "rr0", sh["cell"]), "gz": _require(metrics["gz"], "gz", (nj, ni)),
        "divx": _require(divx, "divx", sh["cell"]), "tendency": _require(tendency, "tendency", sh["cell"]),
    }
    if write_fluxes:
        if fluxes is None:
            raise ValueError("write_fluxes requires the fluxes x/y/z arrays")
        a["flux_x"] = _require(fluxes["x"], "flux_x", sh["u"])
        a["flux_y"] = _require(fluxes["y"], "flux_y", sh["v"])
        a["flux_z"] = _require(fluxes["z"], "flux_z", sh["w"])
    if vertical.flat:
        prof = _require(vertical.mh, "mh", (nk + 2,))
        rdz = float(vertical.rdz)
        if not (math.isfinite(rdz) and rdz > 0.0):
            raise ValueError("a flat column needs rdz > 0")
        col = _VerticalColumn(1, None, prof.data_ptr(), rdz)
    else:
        prof = _require(vertical.rdsf, "rdsf", (nk + 3,))
        col = _VerticalColumn(0, prof.data_ptr(), None, 0.0)
    _no_alias(list(a.values()) + [prof], "stretched scalar inputs, profile, flux scratch, and tendency")
    s = _ScalarAdvArrays(**{n: t.data_ptr() for n, t in a.items()})
    device = a["scalar"].device
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        _native.check(_bind().gm1b_scalar_advection5_column(ni, nj, nk, ctypes.byref(s), nrk, 1 if wflag else 0, dx,
                                                            dy, weps, obc, int(levels_per_chunk or 0),
                                                            ctypes.byref(col), ctypes.c_void_p(st.cuda_stream)),
                      "gm1b_scalar_advection5_column")
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {"operation": "stretched-scalar-advection5", "flat": bool(vertical.flat), "nrk": nrk,
                           "weno": use_weno, "lateral_obc": obc})
