"""The TKE source inputs on B200: deformation (CM1 calcdef) and the moist
squared buoyancy frequency (CM1 calcnm).

Drop-in mirror of the reference operator API (torch CUDA tensors in place of
CuPy arrays; the same array names, shapes, keywords and refusals):

  TerrainDeformationSelection, terrain_deformation_shapes,
  launch_cuda_terrain_deformation     src/cm1core/cuda_terrain_deformation.py:77-157, :914
  MoistNmSelection, moist_nm_array_shapes,
  launch_cuda_moist_nm                src/cm1core/cuda_moist_nm.py:31-131, :542
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

# ------------------------------------------------------------------ calcdef

DEFORMATION_INPUT_NAMES = ("u3d", "v3d", "w3d", "rho", "rf", "c1", "c2", "gz", "rgz", "gzu", "rgzu", "gzv", "rgzv",
                           "gx", "gy")
DEFORMATION_OUTPUT_NAMES = ("defv", "defh")
DEFORMATION_ARRAY_NAMES = DEFORMATION_INPUT_NAMES + DEFORMATION_OUTPUT_NAMES
_DEF_STRUCT = ("u3d", "v3d", "w3d", "rho", "rf", "c1", "c2", "gz", "rgz", "rgzu", "rgzv", "gx", "gy", "defv", "defh")


@dataclass(frozen=True, slots=True)
class TerrainDeformationSelection:
    terrain: bool = True
    axisymmetric: int = 0
    lateral_boundaries: tuple[int, int, int, int] = (2, 2, 2, 2)
    serial_full_domain: bool = True


DEFAULT_TERRAIN_DEFORMATION_SELECTION = TerrainDeformationSelection()


def _grid(ni, nj, nk, minimum_k=3, minimum_h=3) -> None:
    for name, value, minimum in (("ni", ni, minimum_h), ("nj", nj, minimum_h), ("nk", nk, minimum_k)):
        if isinstance(value, bool) or not isinstance(value, int) or value < minimum:
            raise ValueError(f"{name} must be an integer >= {minimum}")


def _positive(name: str, value: Any) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise TypeError(f"{name} must be numeric")
    x = float(value)
    if not math.isfinite(x) or x <= 0.0:
        raise ValueError(f"{name} must be finite and > 0")
    return x


def terrain_deformation_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    _grid(ni, nj, nk)
    cell, face = (nk, nj, ni), (nk + 1, nj, ni)
    return {"u3d": (nk, nj, ni + 1), "v3d": (nk, nj + 1, ni), "w3d": face, "rho": cell, "rf": face, "c1": face,
            "c2": face, "gz": (nj, ni), "rgz": (nj, ni), "gzu": (nj, ni + 1), "rgzu": (nj, ni + 1),
            "gzv": (nj + 1, ni), "rgzv": (nj + 1, ni), "gx": face, "gy": face, "defv": face, "defh": face}


class _DefArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in _DEF_STRUCT]


def _require(arrays: Mapping[str, Any], names, shapes, what: str, dtypes=None) -> dict[str, torch.Tensor]:
    missing = [n for n in names if n not in arrays]
    if missing:
        raise ValueError(f"missing {what} arrays: {', '.join(missing)}")
    out = {}
    for n in names:
        t = arrays[n]
        want = (dtypes or {}).get(n, torch.float32)
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != want or tuple(t.shape) != shapes[n] \
                or not t.is_contiguous():
            raise ValueError(f"{n} must be a contiguous {want} CUDA tensor of shape {shapes[n]}")
        out[n] = t
    if len({t.data_ptr() for t in out.values()}) != len(out):
        raise ValueError(f"{what} arrays must not alias")
    return out


def launch_cuda_terrain_deformation(
    arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float, dz: float,
    selection: TerrainDeformationSelection = DEFAULT_TERRAIN_DEFORMATION_SELECTION, stream: Any | None = None,
) -> CudaLaunch:
    """Enqueue calcdef (terrain, four open sides) without host synchronisation."""
    if not isinstance(selection, TerrainDeformationSelection):
        raise TypeError("selection must be a TerrainDeformationSelection")
    if selection != DEFAULT_TERRAIN_DEFORMATION_SELECTION:
        refuse(code="CM1-CALCDEF-UNSUPPORTED", gate="physics-seam", option="terrain_calcdef_selection",
               value={"terrain": selection.terrain, "axisymmetric": selection.axisymmetric,
                      "lateral_boundaries": list(selection.lateral_boundaries),
                      "serial_full_domain": selection.serial_full_domain},
               reason="only the serial Cartesian terrain branch with four open lateral boundaries is built",
               remedy="use the product selection")
    shapes = terrain_deformation_shapes(ni, nj, nk)
    dx, dy, dz = _positive("dx", dx), _positive("dy", dy), _positive("dz", dz)
    a = _require(arrays, DEFORMATION_ARRAY_NAMES, shapes, "terrain-deformation")
    s = _DefArrays(**{n: a[n].data_ptr() for n in _DEF_STRUCT})
    lib = _native.lib()
    if not getattr(lib, "_def_bound", False):
        i32, f32 = ctypes.c_int32, ctypes.c_float
        lib.gm1b_terrain_deformation.argtypes = [i32, i32, i32, ctypes.POINTER(_DefArrays), f32, f32, f32,
                                                 ctypes.c_void_p]
        lib.gm1b_terrain_deformation.restype = i32
        lib._def_bound = True
    device = a["defv"].device
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        _native.check(lib.gm1b_terrain_deformation(ni, nj, nk, ctypes.byref(s), dx, dy, dz,
                                                   ctypes.c_void_p(st.cuda_stream)), "gm1b_terrain_deformation")
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {"operator": "terrain-calcdef", "live_words": ni * nj * (nk - 1),
                           "boundary_face_zero_words": 2 * ni * nj})


# -------------------------------------------------- calcdef, flat column

FLAT_DEFORMATION_ARRAY_NAMES = ("u3d", "v3d", "w3d", "rho", "rf", "mf", "c1", "c2", "defv", "defh")


class _FlatDefArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("u3d", "v3d", "w3d", "rho", "rf", "mf", "c1", "c2", "mh_profile",
                                               "defv", "defh")]


def flat_deformation_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    _grid(ni, nj, nk)
    cell, face = (nk, nj, ni), (nk + 1, nj, ni)
    return {"u3d": (nk, nj, ni + 1), "v3d": (nk, nj + 1, ni), "w3d": face, "rho": cell, "rf": face, "mf": face,
            "c1": face, "c2": face, "defv": face, "defh": face, "mh_profile": (nk + 2,)}


def launch_cuda_flat_deformation(arrays: Mapping[str, Any], *, mh_profile: Any, ni: int, nj: int, nk: int, dx: float,
                                 dy: float, rdz: float, stream: Any | None = None) -> CudaLaunch:
    """calcdef on a flat (terrain_flag=.false.) stretched column
    (enqueue_flat_calcdef, src/cm1core/cuda_gm1_flat_stretched_closure.py:524,
    with the zero fill of defv/defh of cuda_cartesian_closure.py:1130-1131):
    the strains with rdz*mh(k) (``mh_profile``, nk+2 words, CM1-indexed) and
    rdz*mf(k) (the 3-D face ``mf``), the deformation reduction into defv and
    defh.  ``rdz`` is the vertical coordinate's reference 1/dz."""
    shapes = flat_deformation_shapes(ni, nj, nk)
    dx, dy, rdz = _positive("dx", dx), _positive("dy", dy), _positive("rdz", rdz)
    a = _require({**arrays, "mh_profile": mh_profile}, FLAT_DEFORMATION_ARRAY_NAMES + ("mh_profile",), shapes,
                 "flat-deformation")
    s = _FlatDefArrays(**{f: a[f].data_ptr() for f, _ in _FlatDefArrays._fields_})
    lib = _native.lib()
    if not getattr(lib, "_flatdef_bound", False):
        i32, f32 = ctypes.c_int32, ctypes.c_float
        lib.gm1b_flat_deformation.argtypes = [i32, i32, i32, ctypes.POINTER(_FlatDefArrays), f32, f32, f32,
                                              ctypes.c_void_p]
        lib.gm1b_flat_deformation.restype = i32
        lib._flatdef_bound = True
    device = a["defv"].device
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        _native.check(lib.gm1b_flat_deformation(ni, nj, nk, ctypes.byref(s), dx, dy, rdz,
                                                ctypes.c_void_p(st.cuda_stream)), "gm1b_flat_deformation")
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {"operator": "flat-calcdef", "live_words": ni * nj * (nk - 1),
                           "boundary_face_zero_words": 2 * ni * nj})


# ------------------------------------------------------------------- calcnm

NM_INPUT_NAMES = ("c1", "c2", "mf", "pi0", "th0", "prs", "pp3d", "th3d", "q3d")
NM_FLOAT_OUTPUT_NAMES = ("nm", "temperature", "qt", "thv", "qvci")
NM_MASK_NAME = "saturation_mask"
NM_ARRAY_NAMES = NM_INPUT_NAMES + NM_FLOAT_OUTPUT_NAMES + (NM_MASK_NAME,)


@dataclass(frozen=True, slots=True)
class MoistNmSelection:
    ptype: int = 5
    imoist: int = 1
    iice: int = 1
    numq: int = 6
    nqv: int = 1
    nqc: int = 2
    nqi: int = 4
    nql1: int = 2
    nql2: int = 3
    nqs1: int = 4
    nqs2: int = 6


DEFAULT_MOIST_NM_SELECTION = MoistNmSelection()
_NM_EXPECTED = {
    "physics.native_ptype_context": ("ptype", 5), "physics.moist": ("imoist", 1), "physics.ice": ("iice", 1),
    "physics.moist_species": ("numq", 6), "physics.nqv": ("nqv", 1), "physics.nqc": ("nqc", 2),
    "physics.nqi": ("nqi", 4), "physics.nql1": ("nql1", 2), "physics.nql2": ("nql2", 3),
    "physics.nqs1": ("nqs1", 4), "physics.nqs2": ("nqs2", 6),
}


def moist_nm_array_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    _grid(ni, nj, nk, minimum_k=2, minimum_h=1)
    cell, face = (nk, nj, ni), (nk + 1, nj, ni)
    return {"c1": face, "c2": face, "mf": face, "pi0": (nk,), "th0": (nk,), "prs": cell, "pp3d": cell,
            "th3d": cell, "q3d": (6, nk, nj, ni), "nm": face, "temperature": cell, "qt": cell, "thv": cell,
            "qvci": cell, NM_MASK_NAME: cell}


class _NmArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in NM_ARRAY_NAMES + ("counts",)]


def launch_cuda_moist_nm(
    arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dz: float,
    selection: MoistNmSelection = DEFAULT_MOIST_NM_SELECTION, stream: Any | None = None,
    counts: torch.Tensor | None = None,
) -> CudaLaunch:
    """Enqueue calcnm without host synchronisation.  ``counts`` (four int64
    words, added to) receives the saturated, liquid, mixed and ice face
    counts that the reference's CPU twin returns."""
    if not isinstance(selection, MoistNmSelection):
        raise TypeError("selection must be a MoistNmSelection")
    for option, (attribute, expected) in _NM_EXPECTED.items():
        value = getattr(selection, attribute)
        if isinstance(value, bool) or not isinstance(value, int) or value != expected:
            refuse(code="CM1-MOIST-NM-UNSUPPORTED", gate="physics-seam", option=option, value=value,
                   reason=f"only {option}={expected} is built; another value selects other CM1 species",
                   remedy="use the six-species ice-aware branch")
    shapes = moist_nm_array_shapes(ni, nj, nk)
    dz = _positive("dz", dz)
    a = _require(arrays, NM_ARRAY_NAMES, shapes, "moist-Nm", dtypes={NM_MASK_NAME: torch.uint8})
    ptrs = {n: a[n].data_ptr() for n in NM_ARRAY_NAMES}
    if counts is not None:
        if counts.dtype != torch.int64 or counts.numel() != 4 or not counts.is_cuda:
            raise ValueError("counts must be four int64 CUDA words")
        ptrs["counts"] = counts.data_ptr()
    s = _NmArrays(**ptrs)
    lib = _native.lib()
    if not getattr(lib, "_nm_bound", False):
        i32, f32 = ctypes.c_int32, ctypes.c_float
        lib.gm1b_moist_nm.argtypes = [i32, i32, i32, ctypes.POINTER(_NmArrays), f32, ctypes.c_void_p]
        lib.gm1b_moist_nm.restype = i32
        lib._nm_bound = True
    device = a["nm"].device
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        _native.check(lib.gm1b_moist_nm(ni, nj, nk, ctypes.byref(s), dz, ctypes.c_void_p(st.cuda_stream)),
                      "gm1b_moist_nm")
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {"operator": "moist-nm", "columns": ni * nj, "interior_words": ni * nj * (nk - 1)})
