"""Terrain + all-open psolver=3 acoustic RK stage on B200.

Drop-in mirror of the reference operator API (torch CUDA tensors in place of
CuPy arrays; the same names, keywords, shapes, contracts and errors):

  TerrainOpenSelection, validate_terrain_open_selection
                                   src/cm1core/cuda_terrain_open_boundary.py:108-193
  terrain_static_shapes            :429-459
  TerrainOpenSoundAblations, terrain_open_sound_shapes, COMPARE_OUTPUT_NAMES,
  compare_psolver3_terrain_open_raw
                                   src/cm1core/cuda_psolver3_terrain_open.py:100-188, :276-297, :916-944
  compile_cuda_psolver3_terrain_open(retain_column_diagnostics=)
                                   :1113-1169
  launch_cuda_psolver3_terrain_open_three_stage / _stage
                                   :1217-1432, :1436-1507

Each stage is one library call (gm1b_terrain_open_stage).  The reference's
lateral-family and nest hooks (``lateral``, ``nest_substep``) select code
outside the all-open stage and are refused; ``workspace`` is accepted and
unused (the stage keeps its radiation packing and edge snapshots on chip).
"""

from __future__ import annotations

import ctypes
import hashlib
import math
from dataclasses import dataclass
from typing import Any, Mapping

import numpy as np
import torch

from . import _native
from .errors import refuse

CM1_OPEN_NGXY = 3
CM1_ALPH_F32 = 0.60
CM1_KDIV_F32 = 0.1

PRESSURE_NAMES = ("ppi", "pp3d", "ppx", "ppd", "piadv", "ppterm", "ppten", "thv", "qk", "pk1", "pk2", "mm", "fpk",
                  "divh", "hadvp", "dum3", "elim_c", "elim_d", "tri_aa", "tri_bb", "tri_cc", "tri_dd", "tri_pivot",
                  "tri_residual")
U_NAMES = ("ua", "u3d", "uten", "rru")
V_NAMES = ("va", "v3d", "vten", "rrv")
W_NAMES = ("wa", "w3d", "wten", "rrw")
BOUNDARY_NAMES = ("radbcw", "radbce", "radbcs", "radbcn", "uh", "vh", "ruf", "rvf")
ALL_ARRAY_NAMES = PRESSURE_NAMES + U_NAMES + V_NAMES + W_NAMES + BOUNDARY_NAMES + ("scalar",)
COMPARE_OUTPUT_NAMES = ("u3d", "v3d", "w3d", "pp3d", "ppd", "ppx", "rru", "rrv", "rrw", "radbcw", "radbce", "radbcs",
                        "radbcn", "tri_pivot", "tri_residual")
COLUMN_DIAGNOSTIC_NAMES = ("tri_aa", "tri_bb", "tri_cc", "tri_dd", "tri_pivot", "tri_residual")
TERRAIN_STATIC_REQUIRED = ("terrain_msl", "zh", "zf", "mh", "rmh", "mf", "rmf", "c1", "c2", "rho0_3d", "rr0", "rf0",
                           "rrf0", "gz", "rgz", "gzu", "rgzu", "gzv", "rgzv", "dzdx", "dzdy", "gx", "gxu", "gy", "gyv")
_STRUCT_METRICS = ("rho0_3d", "rr0", "rf0", "rrf0", "c1", "c2", "gz", "rgzu", "rgzv", "dzdx", "dzdy", "gx", "gxu",
                   "gy", "gyv")
_ABLATION_BITS = {"open_consumption": 1, "terrain_pressure_gradient": 2, "transformed_divergence": 4,
                  "pressure_advection": 8, "implicit_vertical_solve": 16, "between_step_pressure_fill": 32,
                  "radiation_history_production": 64, "stage_family_fills": 128}
GM1B_TOS_DIAGNOSTICS = 1


@dataclass(frozen=True, slots=True)
class TerrainOpenSelection:
    psolver: int = 3
    west_boundary: int = 2
    east_boundary: int = 2
    south_boundary: int = 2
    north_boundary: int = 2
    bottom_boundary: int = 1
    top_boundary: int = 1
    hadvordrs: int = 5
    hadvordrv: int = 5
    terrain: bool = True
    mpi: bool = False
    axisymmetric: int = 0
    stretch_x: bool = False
    stretch_y: bool = False
    restricted_outflow: int = 0
    ngxy: int = CM1_OPEN_NGXY
    base_state_policy: str = "broadcast-validation-only"
    source_backed_halos: bool = False
    product_admission: bool = False


DEFAULT_TERRAIN_OPEN_SELECTION = TerrainOpenSelection()
_EXPECTED_SELECTION = {
    "dynamics.psolver": ("psolver", 3), "boundaries.west": ("west_boundary", 2),
    "boundaries.east": ("east_boundary", 2), "boundaries.south": ("south_boundary", 2),
    "boundaries.north": ("north_boundary", 2), "boundaries.bottom": ("bottom_boundary", 1),
    "boundaries.top": ("top_boundary", 1), "advection.hadvordrs": ("hadvordrs", 5),
    "advection.hadvordrv": ("hadvordrv", 5), "grid.terrain": ("terrain", True), "runtime.mpi": ("mpi", False),
    "grid.axisymmetric": ("axisymmetric", 0), "grid.stretch_x": ("stretch_x", False),
    "grid.stretch_y": ("stretch_y", False), "boundaries.restricted_outflow": ("restricted_outflow", 0),
    "grid.ngxy": ("ngxy", CM1_OPEN_NGXY), "base_state.policy": ("base_state_policy", "broadcast-validation-only"),
    "base_state.source_backed_halos": ("source_backed_halos", False),
    "admission.product": ("product_admission", False),
}


def validate_terrain_open_selection(selection: TerrainOpenSelection) -> None:
    """Refuse every branch other than the sealed terrain all-open 5/5 one."""
    if not isinstance(selection, TerrainOpenSelection):
        raise TypeError("selection must be a TerrainOpenSelection")
    for option, (attribute, expected) in _EXPECTED_SELECTION.items():
        value = getattr(selection, attribute)
        if type(value) is not type(expected) or value != expected:
            product = attribute in {"base_state_policy", "source_backed_halos", "product_admission"}
            refuse(code="CM1-TERRAIN-PRODUCT-SEAM-MISSING" if product else "CM1-TERRAIN-OPEN-UNSUPPORTED",
                   gate="dry-dynamics", option=option, value=value,
                   reason=("product admission requires a source-backed terrain hydrostatic base and halo packer"
                           if product else f"only {option}={expected!r} is covered; another value selects other "
                           "CM1 boundary, metric, or advection code"),
                   remedy="use the terrain all-open 5/5 validation profile")


@dataclass(frozen=True, slots=True)
class TerrainOpenSoundAblations:
    open_consumption: bool = True
    terrain_pressure_gradient: bool = True
    transformed_divergence: bool = True
    pressure_advection: bool = True
    implicit_vertical_solve: bool = True
    between_step_pressure_fill: bool = True
    radiation_history_production: bool = True
    stage_family_fills: bool = True


def _ablation_mask(ablations: TerrainOpenSoundAblations) -> int:
    return sum(bit for name, bit in _ABLATION_BITS.items() if getattr(ablations, name))


def terrain_static_shapes(*, ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    for name, value, minimum in (("ni", ni, 3), ("nj", nj, 3), ("nk", nk, 3)):
        if isinstance(value, bool) or not isinstance(value, int) or value < minimum:
            raise ValueError(f"{name} must be an integer >= {minimum}")
    mass, face, plane = (nk, nj, ni), (nk + 1, nj, ni), (nj, ni)
    return {"terrain_msl": plane, "zh": mass, "zf": face, "mh": mass, "rmh": mass, "mf": face, "rmf": face,
            "c1": face, "c2": face, "rho0_3d": mass, "rr0": mass, "rf0": face, "rrf0": face, "gz": plane,
            "rgz": plane, "gzu": (nj, ni + 1), "rgzu": (nj, ni + 1), "gzv": (nj + 1, ni), "rgzv": (nj + 1, ni),
            "dzdx": plane, "dzdy": plane, "gx": face, "gxu": (nk + 1, nj, ni + 1), "gy": face,
            "gyv": (nk + 1, nj + 1, ni)}


def terrain_open_sound_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    terrain_static_shapes(ni=ni, nj=nj, nk=nk)
    ng = CM1_OPEN_NGXY
    shapes: dict[str, tuple[int, ...]] = {n: (nk + 2, nj + 2, ni + 2) for n in PRESSURE_NAMES}
    shapes.update({n: (nk + 2, nj + 2 * ng, ni + 1 + 2 * ng) for n in U_NAMES})
    shapes.update({n: (nk + 2, nj + 1 + 2 * ng, ni + 2 * ng) for n in V_NAMES})
    shapes.update({n: (nk + 3, nj + 2 * ng, ni + 2 * ng) for n in W_NAMES})
    shapes.update({"radbcw": (nk + 2, nj + 2 * ng), "radbce": (nk + 2, nj + 2 * ng),
                   "radbcs": (nk + 2, ni + 2 * ng), "radbcn": (nk + 2, ni + 2 * ng), "uh": (ni + 2 * ng,),
                   "vh": (nj + 2 * ng,), "ruf": (ni + 1 + 2 * ng,), "rvf": (nj + 1 + 2 * ng,),
                   "scalar": (nk + 2, nj + 2 * ng, ni + 2 * ng)})
    return shapes


def compare_psolver3_terrain_open_raw(expected: Mapping[str, Any], candidate: Mapping[str, Any]) -> dict[str, Any]:
    """Compare every declared output with raw-bit, no-null semantics (host
    numpy arrays, or tensors that are copied to the host)."""
    out: dict[str, Any] = {}
    for name in COMPARE_OUTPUT_NAMES:
        if name not in expected or name not in candidate:
            raise ValueError(f"missing terrain/open comparison output {name}")
        left, right = (x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else x
                       for x in (expected[name], candidate[name]))
        if not isinstance(left, np.ndarray) or not isinstance(right, np.ndarray):
            raise TypeError(f"{name} comparison values must be numpy.ndarray")
        if left.dtype != np.float32 or right.dtype != np.float32 or left.shape != right.shape:
            raise ValueError(f"{name} comparison dtype/shape mismatch")
        out[name] = {"exact": bool(np.array_equal(left.view(np.uint32), right.view(np.uint32))),
                     "expected_sha256": hashlib.sha256(left.tobytes(order="C")).hexdigest(),
                     "candidate_sha256": hashlib.sha256(right.tobytes(order="C")).hexdigest()}
    return {"mode": "raw-bit", "max_ulp": 0, "null_or_missing_is_pass": False,
            "passed": all(v["exact"] for v in out.values()), "fields": out}


class _Arrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ALL_ARRAY_NAMES]


class _Metrics(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in _STRUCT_METRICS]


def _lib():
    lib = _native.lib()
    if not getattr(lib, "_tos_bound", False):
        c = ctypes
        lib.gm1b_terrain_open_stage.argtypes = [c.c_int32] * 4 + [c.c_float, c.c_int32, c.c_float, c.c_float,
                                                                  c.c_double, c.c_float, c.c_float, c.c_uint32,
                                                                  c.c_uint32, c.POINTER(_Arrays),
                                                                  c.POINTER(_Metrics), c.c_void_p]
        lib.gm1b_terrain_open_stage.restype = c.c_int32
        from .momentum import _Column
        lib.gm1b_terrain_open_stage_column.argtypes = [c.c_int32] * 4 + [c.c_float, c.c_int32, c.c_float, c.c_float,
                                                                         c.c_float, c.c_float, c.c_uint32,
                                                                         c.c_uint32, c.c_uint32, c.POINTER(_Arrays),
                                                                         c.POINTER(_Metrics), c.POINTER(_Column),
                                                                         c.c_void_p]
        lib.gm1b_terrain_open_stage_column.restype = c.c_int32
        lib._tos_bound = True
    return lib


@dataclass(frozen=True, slots=True)
class CompiledPsolver3TerrainOpenKernels:
    """The in-tree library's terrain/open stage entry, with the diagnostic
    retention the reference binds at compile time."""
    retain_column_diagnostics: bool = True
    entry: str = "gm1b_terrain_open_stage"


def compile_cuda_psolver3_terrain_open(*, retain_column_diagnostics: bool = True) -> CompiledPsolver3TerrainOpenKernels:
    if type(retain_column_diagnostics) is not bool:
        raise TypeError("retain_column_diagnostics must be bool")
    _lib()
    return CompiledPsolver3TerrainOpenKernels(retain_column_diagnostics)


@dataclass(frozen=True, slots=True)
class CudaPsolver3TerrainOpenLaunch:
    ready_event: Any
    compiled: CompiledPsolver3TerrainOpenKernels
    cadence: tuple[dict[str, Any], ...]
    receipt: dict[str, Any]


def _positive(name: str, value: Any) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise TypeError(f"{name} must be numeric")
    x = float(value)
    if not math.isfinite(x) or x <= 0.0:
        raise ValueError(f"{name} must be finite and > 0")
    return x


def _require_device_arrays(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int,
                           retain_column_diagnostics: bool) -> dict[str, torch.Tensor]:
    shapes = terrain_open_sound_shapes(ni, nj, nk)
    if not retain_column_diagnostics:
        shapes.update({name: (1,) for name in COLUMN_DIAGNOSTIC_NAMES})
    missing = [n for n in ALL_ARRAY_NAMES if n not in arrays]
    if missing:
        raise ValueError(f"missing CUDA terrain/open sound arrays: {', '.join(missing)}")
    out = {}
    for n in ALL_ARRAY_NAMES:
        t = arrays[n]
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 \
                or tuple(t.shape) != shapes[n] or not t.is_contiguous():
            raise ValueError(f"CUDA terrain/open sound {n} has invalid dtype, shape, or layout")
        out[n] = t
    if len({t.data_ptr() for t in out.values()}) != len(out):
        raise ValueError("CUDA terrain/open sound arrays must not alias")
    return out


def _require_device_metrics(metrics: Mapping[str, Any], *, ni: int, nj: int, nk: int) -> dict[str, torch.Tensor]:
    shapes = terrain_static_shapes(ni=ni, nj=nj, nk=nk)
    missing = [n for n in TERRAIN_STATIC_REQUIRED if n not in metrics]
    if missing:
        raise ValueError(f"missing CUDA terrain/open metrics: {', '.join(missing)}")
    out = {}
    for n in TERRAIN_STATIC_REQUIRED:
        t = metrics[n]
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 \
                or tuple(t.shape) != shapes[n] or not t.is_contiguous():
            raise ValueError(f"CUDA terrain/open metric {n} has invalid dtype, shape, or layout")
        out[n] = t
    return out


def launch_cuda_psolver3_terrain_open_three_stage(
        arrays: Mapping[str, Any], metrics: Mapping[str, Any], *, ni: int, nj: int, nk: int, dt: float, nsound: int,
        dx: float, dy: float, dz: float, selection: TerrainOpenSelection = DEFAULT_TERRAIN_OPEN_SELECTION,
        ablations: TerrainOpenSoundAblations | None = None, stream: Any | None = None,
        compiled: CompiledPsolver3TerrainOpenKernels | None = None, terrain_compiled: Any | None = None,
        open_compiled: Any | None = None, lateral_compiled: Any | None = None, lateral: Any | None = None,
        workspace: Mapping[str, Any] | None = None, alph: float | None = None, kdiv: float | None = None,
        _nrk_sequence: tuple[int, ...] = (1, 2, 3), nest_substep: Any | None = None) -> CudaPsolver3TerrainOpenLaunch:
    """Enqueue the source-ordered terrain/open acoustic stages on ``stream``
    (the current stream when None); ``alph`` / ``kdiv`` default to CM1's
    0.60 and 0.10."""
    from .periodic import sound3_stage_schedule_f32

    del terrain_compiled, open_compiled, lateral_compiled, workspace
    validate_terrain_open_selection(selection)
    for name, value in (("alph", alph), ("kdiv", kdiv)):
        if value is None:
            continue
        if isinstance(value, bool) or not isinstance(value, (int, float)):
            raise TypeError(f"{name} must be numeric or None")
        if not (0.0 <= float(value) <= 1.0):
            raise ValueError(f"{name}={value} is outside CM1's admitted [0, 1]")
    if _nrk_sequence not in ((1, 2, 3), (1,), (2,), (3,)):
        raise ValueError("internal terrain/open acoustic sequence must be (1,2,3) or one explicit RK stage")
    dt, dx, dy, dz = (_positive(n, v) for n, v in (("dt", dt), ("dx", dx), ("dy", dy), ("dz", dz)))
    if ablations is None:
        ablations = TerrainOpenSoundAblations()
    if not isinstance(ablations, TerrainOpenSoundAblations):
        raise TypeError("ablations must be TerrainOpenSoundAblations")
    if lateral is not None:
        refuse(code="CM1-TERRAIN-LATERAL-FAMILY", gate="dry-dynamics", option="lateral", value=type(lateral).__name__,
               reason="periodic, rigid and Klemp-Wilhelmson lateral families replace the all-open consumption and "
                      "radiation this stage computes", remedy="run the all-open stage (lateral=None)")
    if nest_substep is not None:
        refuse(code="CM1-TERRAIN-NEST-SUBSTEP", gate="dry-dynamics", option="nest_substep",
               value=type(nest_substep).__name__, reason="a nest's specified zone edits the state between the "
               "phases of every small step", remedy="run the stage without a live nest")
    compiled = compiled or compile_cuda_psolver3_terrain_open()
    if not isinstance(compiled, CompiledPsolver3TerrainOpenKernels):
        raise TypeError("compiled must come from compile_cuda_psolver3_terrain_open")
    retain = compiled.retain_column_diagnostics
    a = _require_device_arrays(arrays, ni=ni, nj=nj, nk=nk, retain_column_diagnostics=retain)
    m = _require_device_metrics(metrics, ni=ni, nj=nj, nk=nk)
    device = a["u3d"].device
    if any(t.device != device for t in (*a.values(), *m.values())):
        raise ValueError("terrain/open arrays and metrics must live on one CUDA device")
    alph32 = float(np.float32(CM1_ALPH_F32 if alph is None else alph))
    kdiv32 = float(np.float32(CM1_KDIV_F32 if kdiv is None else kdiv))
    mask = _ablation_mask(ablations)
    lib = _lib()
    st = torch.cuda.current_stream(device) if stream is None else stream
    sa = _Arrays(**{n: a[n].data_ptr() for n in ALL_ARRAY_NAMES})
    sm = _Metrics(**{n: m[n].data_ptr() for n in _STRUCT_METRICS})
    cadence = []
    with torch.cuda.device(device), torch.cuda.stream(st):
        for nrk in _nrk_sequence:
            nloop, dts = sound3_stage_schedule_f32(dt, nsound, nrk)
            _native.check(lib.gm1b_terrain_open_stage(ni, nj, nk, nrk, dt, nsound, dx, dy, dz, alph32, kdiv32, mask,
                                                      GM1B_TOS_DIAGNOSTICS if retain else 0, ctypes.byref(sa),
                                                      ctypes.byref(sm), ctypes.c_void_p(st.cuda_stream)),
                          "gm1b_terrain_open_stage")
            cadence.append({"nrk": nrk, "nloop": nloop, "dts_f32": float(dts),
                            "open_consumptions": nloop if ablations.open_consumption else 0,
                            "pressure_fills": nloop - 1 if ablations.between_step_pressure_fill else 0,
                            "radiation_productions": 1 if ablations.radiation_history_production else 0})
        event = torch.cuda.Event()
        event.record(st)
    receipt: dict[str, Any] = {
        "domain": {"ni": ni, "nj": nj, "nk": nk, "ngxy": CM1_OPEN_NGXY},
        "cadence": cadence,
        "acoustic_reals": {"alph": alph32, "kdiv": kdiv32},
        "comparison_contract": {"mode": "raw-bit", "max_ulp": 0, "null_or_missing_is_pass": False},
        "lateral_boundaries": {"selection": {"wbc": 2, "ebc": 2, "sbc": 2, "nbc": 2, "irbc": 4, "roflux": 0,
                                             "nudgeobc": 0}},
        "launches_per_stage": "1 + 3*nloop + 3",
    }
    if not retain:
        receipt["column_diagnostics"] = {"retained": False, "omitted_arrays": list(COLUMN_DIAGNOSTIC_NAMES) + [
            "fpk", "divh", "hadvp", "dum3", "elim_c", "elim_d"]}
    return CudaPsolver3TerrainOpenLaunch(event, compiled, tuple(cadence), receipt)


def launch_cuda_psolver3_terrain_open_stage(arrays: Mapping[str, Any], metrics: Mapping[str, Any], *, ni: int, nj: int,
                                            nk: int, nrk: int, dt: float, nsound: int, dx: float, dy: float,
                                            dz: float, **kwargs: Any) -> CudaPsolver3TerrainOpenLaunch:
    """Enqueue exactly one acoustic RK stage."""
    if isinstance(nrk, bool) or not isinstance(nrk, int) or nrk not in (1, 2, 3):
        raise ValueError("nrk must select explicit CM1 RK stage 1, 2, or 3")
    if "_nrk_sequence" in kwargs:
        raise TypeError("launch_cuda_psolver3_terrain_open_stage takes nrk, not _nrk_sequence")
    launch = launch_cuda_psolver3_terrain_open_three_stage(arrays, metrics, ni=ni, nj=nj, nk=nk, dt=dt, nsound=nsound,
                                                           dx=dx, dy=dy, dz=dz, _nrk_sequence=(nrk,), **kwargs)
    receipt = {**launch.receipt, "nrk": nrk, "three_stage_composition": False}
    return CudaPsolver3TerrainOpenLaunch(launch.ready_event, launch.compiled, launch.cadence, receipt)


def launch_cuda_gm1_child_psolver3_open_stage(
        arrays: Mapping[str, Any], metrics: Mapping[str, Any], *, ni: int, nj: int, nk: int, nrk: int, dt: float,
        nsound: int, dx: float, dy: float, vertical: Any, selection: TerrainOpenSelection = DEFAULT_TERRAIN_OPEN_SELECTION,
        ablations: TerrainOpenSoundAblations | None = None, stream: Any | None = None,
        compiled: CompiledPsolver3TerrainOpenKernels | None = None, alph: float | None = None,
        kdiv: float | None = None, lateral_sides: tuple[int, int, int, int] = (2, 2, 2, 2),
        **unused: Any) -> CudaPsolver3TerrainOpenLaunch:
    """Enqueue one acoustic RK stage on a stretched column
    (src/cm1core/cuda_gm1_child_psolver3_open.py:848).  ``vertical`` is a
    :class:`gm1_b200.momentum.StretchedMomentumColumn`.  Terrain column
    (``flat=False``): its ``sigma`` (nk+2), ``sigmaf`` (nk+3), ``rds`` (nk+2),
    ``rdsf`` (nk+3) and the lid ``ztop``, which must be the column's own
    sigmaf(nk+1) (param.F:8193); the stage is sealed to four open sides.
    Flat column (``flat=True``): sound.F's terrain_flag=.false. statements on
    ``mh`` (nk+2), ``mf`` (nk+3) and ``rdz``, with ``lateral_sides`` as
    sound.F takes it (the pressure gradient's dtu0/dtv0 mask, ssopenbc on
    the open sides only).  ``metrics`` carries the 25 terrain metrics and
    ``rho0_padded`` (nk+2, nj+6, ni+6), the source-valid padded base density
    whose face averages weight the terrain column's pressure advection.
    There is no dz: every vertical derivative reads the profiles."""
    from .momentum import StretchedMomentumColumn, _Column, momentum_lateral_sides, momentum_open_boundary_code
    from .periodic import sound3_stage_schedule_f32

    for name in unused:
        if name not in ("open_compiled", "lateral_compiled", "workspace", "allow_compact_validation",
                        "allow_uniform_idealized_validation", "nest_substep"):
            raise TypeError(f"unexpected keyword {name!r}")
    if unused.get("nest_substep") is not None:
        refuse(code="CM1-TERRAIN-NEST-SUBSTEP", gate="dry-dynamics", option="nest_substep",
               value=type(unused["nest_substep"]).__name__, reason="a nest's specified zone edits the state between "
               "the phases of every small step", remedy="run the stage without a live nest")
    validate_terrain_open_selection(selection)
    if not isinstance(vertical, StretchedMomentumColumn):
        raise TypeError("vertical must be a StretchedMomentumColumn")
    flat = bool(vertical.flat)
    obc = momentum_open_boundary_code(lateral_sides)
    if not flat and tuple(lateral_sides) != (2, 2, 2, 2):
        raise ValueError(f"lateral_sides {tuple(lateral_sides)}: the terrain child acoustic stage runs bc.F's ssopenbc "
                         "on all four sides and its pressure gradient skips every boundary face")
    for name, value in (("alph", alph), ("kdiv", kdiv)):
        if value is None:
            continue
        if isinstance(value, bool) or not isinstance(value, (int, float)):
            raise TypeError(f"{name} must be numeric or None")
        if not (0.0 <= float(value) <= 1.0):
            raise ValueError(f"{name}={value} is outside CM1's admitted [0, 1]")
    for name, value in (("ni", ni), ("nj", nj), ("nk", nk)):
        if isinstance(value, bool) or not isinstance(value, int):
            raise ValueError(f"{name} must be an integer")
    if nk < 4:
        raise ValueError("child psolver requires nk >= 4; param.F:8985-9060 extrapolates from four scalar levels at "
                         "each end of the column")
    if ni < 3 or nj < 3:
        raise ValueError("child psolver requires ni,nj >= 3")
    if isinstance(nrk, bool) or not isinstance(nrk, int) or nrk not in (1, 2, 3):
        raise ValueError("nrk must be 1, 2, or 3")
    dt, dx, dy = (_positive(n, v) for n, v in (("dt", dt), ("dx", dx), ("dy", dy)))
    if isinstance(nsound, bool) or not isinstance(nsound, int) or nsound < 1:
        raise ValueError("nsound must be a positive integer")
    if ablations is None:
        ablations = TerrainOpenSoundAblations()
    if not isinstance(ablations, TerrainOpenSoundAblations):
        raise TypeError("ablations must be TerrainOpenSoundAblations")
    compiled = compiled or compile_cuda_psolver3_terrain_open()
    if not isinstance(compiled, CompiledPsolver3TerrainOpenKernels):
        raise TypeError("compiled must come from compile_cuda_psolver3_terrain_open")
    retain = compiled.retain_column_diagnostics
    a = _require_device_arrays(arrays, ni=ni, nj=nj, nk=nk, retain_column_diagnostics=retain)
    m = _require_device_metrics(metrics, ni=ni, nj=nj, nk=nk)
    if "rho0_padded" not in metrics:
        raise ValueError("metrics must expose source-valid padded rho0 as rho0_padded; physical rho0_3d cannot "
                         "source outer-face averages")
    rho0p = metrics["rho0_padded"]
    shape = (nk + 2, nj + 6, ni + 6)
    if not (isinstance(rho0p, torch.Tensor) and rho0p.is_cuda and rho0p.dtype == torch.float32
            and tuple(rho0p.shape) == shape and rho0p.is_contiguous()):
        raise ValueError(f"rho0_padded must be device C-f32 {shape}")
    if any(rho0p.data_ptr() == t.data_ptr() for t in a.values()):
        raise ValueError("rho0_padded must not alias a mutable acoustic array")
    prof = {}
    names = (("mh", (nk + 2,)), ("mf", (nk + 3,))) if flat else \
        (("sigma", (nk + 2,)), ("sigmaf", (nk + 3,)), ("rds", (nk + 2,)), ("rdsf", (nk + 3,)))
    for n, pshape in names:
        t = getattr(vertical, n)
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32
                and tuple(t.shape) == pshape and t.is_contiguous()):
            raise ValueError(f"vertical {n} must be device C-f32 {pshape}")
        prof[n] = t
    if len({t.data_ptr() for t in prof.values()}) != len(prof):
        raise ValueError("vertical profiles must not alias")
    ztop = rdz = 0.0
    if flat:
        rdz = float(np.float32(vertical.rdz))
        if not (math.isfinite(rdz) and rdz > 0.0):
            raise ValueError("a flat column needs rdz > 0")
    else:
        ztop = float(np.float32(vertical.ztop))
        if not (math.isfinite(ztop) and ztop > 0.0):
            raise ValueError("vertical top must be finite and greater than zero")
        top_face = float(prof["sigmaf"][nk + 1].item())
        if top_face != ztop:
            raise ValueError(f"vertical top {ztop} m is not this coordinate's own sigmaf(nk+1) of {top_face} m "
                             "(param.F:8193)")
    device = a["u3d"].device
    if any(t.device != device for t in (*a.values(), *m.values(), rho0p, *prof.values())):
        raise ValueError("terrain/open arrays, metrics and profiles must live on one CUDA device")
    alph32 = float(np.float32(CM1_ALPH_F32 if alph is None else alph))
    kdiv32 = float(np.float32(CM1_KDIV_F32 if kdiv is None else kdiv))
    mask = _ablation_mask(ablations)
    lib = _lib()
    st = torch.cuda.current_stream(device) if stream is None else stream
    sa = _Arrays(**{n: a[n].data_ptr() for n in ALL_ARRAY_NAMES})
    sm = _Metrics(**{n: m[n].data_ptr() for n in _STRUCT_METRICS})
    if flat:
        col = _Column(1, rho0p.data_ptr(), None, None, None, None, 0.0, prof["mh"].data_ptr(), prof["mf"].data_ptr(),
                      None, rdz)
    else:
        col = _Column(0, rho0p.data_ptr(), prof["sigma"].data_ptr(), prof["sigmaf"].data_ptr(),
                      prof["rds"].data_ptr(), prof["rdsf"].data_ptr(), ztop, None, None, None, 0.0)
    nloop, dts = sound3_stage_schedule_f32(dt, nsound, nrk)
    with torch.cuda.device(device), torch.cuda.stream(st):
        _native.check(lib.gm1b_terrain_open_stage_column(ni, nj, nk, nrk, dt, nsound, dx, dy, alph32, kdiv32, mask,
                                                         GM1B_TOS_DIAGNOSTICS if retain else 0, obc, ctypes.byref(sa),
                                                         ctypes.byref(sm), ctypes.byref(col),
                                                         ctypes.c_void_p(st.cuda_stream)),
                      "gm1b_terrain_open_stage_column")
        event = torch.cuda.Event()
        event.record(st)
    cadence = ({"nrk": nrk, "nloop": nloop, "dts_f32": float(dts),
                "open_consumptions": nloop if ablations.open_consumption else 0,
                "pressure_fills": nloop - 1 if ablations.between_step_pressure_fill else 0,
                "radiation_productions": 1 if ablations.radiation_history_production else 0},)
    receipt: dict[str, Any] = {
        "domain": {"ni": ni, "nj": nj, "nk": nk, "ngxy": CM1_OPEN_NGXY},
        "vertical": {"branch": "flat" if flat else "terrain", "ztop_f32": None if flat else ztop,
                     "rdz_f32": rdz if flat else None, "dz": None},
        "cadence": list(cadence), "nrk": nrk,
        "acoustic_reals": {"alph": alph32, "kdiv": kdiv32},
        "comparison_contract": {"mode": "raw-bit", "max_ulp": 0, "null_or_missing_is_pass": False},
        "lateral_boundaries": {"selection": dict(zip(("wbc", "ebc", "sbc", "nbc"),
                                                     momentum_lateral_sides(lateral_sides)))},
    }
    return CudaPsolver3TerrainOpenLaunch(event, compiled, cadence, receipt)
