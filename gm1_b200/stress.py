"""The SGS stress of the flat (terrain_flag=.false.) stretched column on
B200: CM1 gettau and the momentum stress divergence turbu/turbv/turbw.

Drop-in mirror of the reference operator API (torch CUDA tensors in place of
CuPy arrays; the same array names and shapes; the two-part binding is not
built and is refused):

  launch_cuda_flat_strain          the strain half of enqueue_flat_calcdef
                                   src/cm1core/cuda_gm1_flat_stretched_closure.py:524
  launch_cuda_flat_gettau          enqueue_flat_gettau           :551
  launch_cuda_flat_momentum_stress enqueue_flat_momentum_stress  :574
  launch_cuda_flat_sgs_stress      the three in order (the stress block of
                                   cuda_cartesian_closure.py:1293-1317)

Each enqueues on ``stream`` (default: the current stream) and returns at
once; the tendencies are ADDED into uten, vten and wten.
"""

from __future__ import annotations

import ctypes
from typing import Any, Mapping

import torch

from . import _native
from .closure import _grid, _positive, _require
from .errors import refuse
from .periodic import CudaLaunch

_FIELDS = ("u3d", "v3d", "w3d", "rho", "rf", "mh", "mf", "mh_profile", "kmh", "kmv", "s11", "s22", "s33", "s12",
           "s13", "s23", "t11", "t22", "t33", "t12", "t13", "t23", "uten", "vten", "wten")
STRAIN_NAMES = ("s11", "s22", "s33", "s12", "s13", "s23")
TAU_NAMES = ("t11", "t22", "t33", "t12", "t13", "t23")
STRAIN_ARRAY_NAMES = ("u3d", "v3d", "w3d", "rho", "rf", "mf", "mh_profile") + STRAIN_NAMES
GETTAU_ARRAY_NAMES = STRAIN_NAMES + ("kmh", "kmv") + TAU_NAMES
MOMENTUM_STRESS_ARRAY_NAMES = TAU_NAMES + ("kmh", "kmv", "rho", "rf", "mh", "mf", "u3d", "v3d", "w3d", "uten",
                                           "vten", "wten")
SGS_STRESS_ARRAY_NAMES = tuple(dict.fromkeys(STRAIN_ARRAY_NAMES + GETTAU_ARRAY_NAMES + MOMENTUM_STRESS_ARRAY_NAMES))
MAX_NK = 200


class _Arrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in _FIELDS]


def flat_stress_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    _grid(ni, nj, nk)
    cell, face = (nk, nj, ni), (nk + 1, nj, ni)
    return {"u3d": (nk, nj, ni + 1), "v3d": (nk, nj + 1, ni), "w3d": face, "rho": cell, "rf": face, "mh": cell,
            "mf": face, "mh_profile": (nk + 2,), "kmh": face, "kmv": face,
            **{n: cell for n in ("s11", "s22", "s33", "t11", "t22", "t33")},
            "s12": (nk, nj + 1, ni + 1), "t12": (nk, nj + 1, ni + 1), "s13": (nk + 1, nj, ni + 1),
            "t13": (nk + 1, nj, ni + 1), "s23": (nk + 1, nj + 1, ni), "t23": (nk + 1, nj + 1, ni),
            "uten": (nk, nj, ni + 1), "vten": (nk, nj + 1, ni), "wten": face}


def _bind(lib) -> None:
    if getattr(lib, "_stress_bound", False):
        return
    i32, f32, vp = ctypes.c_int32, ctypes.c_float, ctypes.c_void_p
    a = ctypes.POINTER(_Arrays)
    lib.gm1b_flat_strain.argtypes = [i32, i32, i32, a, f32, f32, f32, vp]
    lib.gm1b_flat_gettau.argtypes = [i32, i32, i32, a, vp]
    lib.gm1b_flat_momentum_stress.argtypes = [i32, i32, i32, a, f32, f32, f32, f32, vp]
    lib.gm1b_flat_sgs_stress.argtypes = [i32, i32, i32, a, f32, f32, f32, f32, vp]
    for n in ("gm1b_flat_strain", "gm1b_flat_gettau", "gm1b_flat_momentum_stress", "gm1b_flat_sgs_stress"):
        getattr(lib, n).restype = i32
    lib._stress_bound = True


def _prepare(arrays: Mapping[str, Any], names, ni, nj, nk, what):
    _grid(ni, nj, nk)
    if nk > MAX_NK:
        raise ValueError(f"nk must be <= {MAX_NK} (the column solves' shared memory)")
    a = _require(arrays, names, flat_stress_shapes(ni, nj, nk), what)
    s = _Arrays(**{n: (a[n].data_ptr() if n in a else None) for n in _FIELDS})
    lib = _native.lib()
    _bind(lib)
    return a, s, lib


def _launch(a, fn, args, name, record) -> CudaLaunch:
    device = next(iter(a.values())).device
    st = torch.cuda.current_stream(device) if record["stream"] is None else record["stream"]
    with torch.cuda.device(device):
        _native.check(fn(*args, ctypes.c_void_p(st.cuda_stream)), name)
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, record["receipt"])


def launch_cuda_flat_strain(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float,
                            rdz: float, stream: Any | None = None) -> CudaLaunch:
    """The strain carriers rho*Sij of the flat calcdef (gm1_flat_calcdef_mass_v1
    and _face_v1): s11/s22/s33 at cells, s12 at every corner, s13/s23 on face
    levels 1..nk-1.  ``mh_profile`` (nk+2 words, CM1-indexed) and the 3-D
    face ``mf`` carry the stretching; ``rdz`` is the coordinate's 1/dz."""
    dx, dy, rdz = _positive("dx", dx), _positive("dy", dy), _positive("rdz", rdz)
    a, s, lib = _prepare(arrays, STRAIN_ARRAY_NAMES, ni, nj, nk, "flat-strain")
    return _launch(a, lib.gm1b_flat_strain, (ni, nj, nk, ctypes.byref(s), dx, dy, rdz), "gm1b_flat_strain",
                   {"stream": stream, "receipt": {"operator": "flat-strain", "cell_words": ni * nj * nk}})


def launch_cuda_flat_gettau(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int,
                            stream: Any | None = None) -> CudaLaunch:
    """gettau with the free-slip lower and upper faces (enqueue_flat_gettau)."""
    a, s, lib = _prepare(arrays, GETTAU_ARRAY_NAMES, ni, nj, nk, "flat-gettau")
    return _launch(a, lib.gm1b_flat_gettau, (ni, nj, nk, ctypes.byref(s)), "gm1b_flat_gettau",
                   {"stream": stream, "receipt": {"operator": "flat-gettau",
                                                  "stress_words": nk * (3 * ni * nj + (ni + 1) * (nj + 1)) +
                                                  (nk + 1) * ((ni + 1) * nj + ni * (nj + 1))}})


def launch_cuda_flat_momentum_stress(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float,
                                     rdz: float, dt: float, two_part: Any = None,
                                     stream: Any | None = None) -> CudaLaunch:
    """turbu, turbv and turbw with their implicit vertical solves added into
    uten, vten and wten (enqueue_flat_momentum_stress).  The two-part
    (sgsmodel 3/4) binding is not built."""
    if two_part is not None:
        refuse(code="CM1-SGS-STRESS-TWO-PART", gate="physics-seam", option="two_part", value="bound",
               reason="the two-part dot2p block of turbuz/turbvz is not built on this path",
               remedy="run sgsmodel 1 (two_part=None)")
    dx, dy, rdz, dt = _positive("dx", dx), _positive("dy", dy), _positive("rdz", rdz), _positive("dt", dt)
    a, s, lib = _prepare(arrays, MOMENTUM_STRESS_ARRAY_NAMES, ni, nj, nk, "flat-momentum-stress")
    return _launch(a, lib.gm1b_flat_momentum_stress, (ni, nj, nk, ctypes.byref(s), dx, dy, rdz, dt),
                   "gm1b_flat_momentum_stress",
                   {"stream": stream, "receipt": {"operator": "flat-momentum-stress",
                                                  "u_tendency_words": nk * nj * (ni + 1),
                                                  "v_tendency_words": nk * (nj + 1) * ni,
                                                  "w_tendency_words": (nk - 1) * nj * ni}})


def launch_cuda_flat_sgs_stress(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float,
                                rdz: float, dt: float, stream: Any | None = None) -> CudaLaunch:
    """The strain carriers, gettau and the momentum stress in that order."""
    dx, dy, rdz, dt = _positive("dx", dx), _positive("dy", dy), _positive("rdz", rdz), _positive("dt", dt)
    a, s, lib = _prepare(arrays, SGS_STRESS_ARRAY_NAMES, ni, nj, nk, "flat-sgs-stress")
    return _launch(a, lib.gm1b_flat_sgs_stress, (ni, nj, nk, ctypes.byref(s), dx, dy, rdz, dt),
                   "gm1b_flat_sgs_stress", {"stream": stream, "receipt": {"operator": "flat-sgs-stress"}})


# ------------------------------------------------------------ turbs (flat)

SCALAR_TURBULENCE_ARRAY_NAMES = ("th0", "tha", "qa", "rho", "rr", "rf", "mh", "mf", "khh", "khv", "thten1", "qten",
                                 "workspace")


class _TurbsArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("th0", "tha", "qa", "rho", "rr", "rf", "mh", "mf", "khh", "khv",
                                               "thten", "qten", "workspace")]


def scalar_turbulence_workspace(ni: int, nj: int, nk: int, numq: int, device) -> torch.Tensor:
    """The device scratch launch_cuda_flat_scalar_turbulence takes as
    ``workspace``: the horizontal flux divergence of each of the 1 + numq
    scalars."""
    return torch.empty((numq + 1, nk, nj, ni), dtype=torch.float32, device=device)


def flat_scalar_turbulence_shapes(ni: int, nj: int, nk: int, numq: int) -> dict[str, tuple[int, ...]]:
    _grid(ni, nj, nk)
    cell, face = (nk, nj, ni), (nk + 1, nj, ni)
    return {"th0": (nk,), "tha": cell, "qa": (numq, nk, nj, ni), "rho": cell, "rr": cell, "rf": face, "mh": cell,
            "mf": face, "khh": face, "khv": face, "thten1": cell, "qten": (numq, nk, nj, ni),
            "workspace": (numq + 1, nk, nj, ni)}


def launch_cuda_flat_scalar_turbulence(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, numq: int,
                                       dx: float, dy: float, dz: float, dt: float,
                                       stream: Any | None = None) -> CudaLaunch:
    """turbs on the flat stretched column: theta ((th0 - 300) + tha) into
    ``thten1``, then moisture rows 0..numq-1 of ``qa`` into those of
    ``qten`` (added), with khh across the open-halo copies and the implicit
    vertical diffusion with khv, zero surface flux (the scalar loop of the
    closure's held phase on the flat lane, cuda_cartesian_closure.py:1566-1633).
    ``qa`` and ``qten`` may hold more rows than numq (leading rows used);
    ``workspace`` is scalar_turbulence_workspace()'s scratch; ``dz`` is the
    coordinate's reference spacing."""
    if isinstance(numq, bool) or not isinstance(numq, int) or not 0 <= numq <= 6:
        raise ValueError("numq must be an integer in 0..6")
    dx, dy, dz, dt = _positive("dx", dx), _positive("dy", dy), _positive("dz", dz), _positive("dt", dt)
    _grid(ni, nj, nk)
    if nk > MAX_NK:
        raise ValueError(f"nk must be <= {MAX_NK} (the column solve's shared memory)")
    shapes = flat_scalar_turbulence_shapes(ni, nj, nk, numq)
    for n in ("qa", "qten"):
        t = arrays.get(n)
        if isinstance(t, torch.Tensor) and t.dim() == 4 and t.shape[0] >= numq:
            shapes[n] = tuple(t.shape)
    a = _require(arrays, SCALAR_TURBULENCE_ARRAY_NAMES, shapes, "flat-scalar-turbulence")
    if tuple(a["qa"].shape[1:]) != (nk, nj, ni) or tuple(a["qten"].shape[1:]) != (nk, nj, ni):
        raise ValueError("qa and qten must hold rows of shape (nk, nj, ni)")
    s = _TurbsArrays(**{f: a["thten1" if f == "thten" else f].data_ptr() for f, _ in _TurbsArrays._fields_})
    lib = _native.lib()
    if not getattr(lib, "_turbs_bound", False):
        i32, f32 = ctypes.c_int32, ctypes.c_float
        lib.gm1b_flat_scalar_turbulence.argtypes = [i32, i32, i32, i32, ctypes.POINTER(_TurbsArrays), f32, f32, f32,
                                                    f32, ctypes.c_void_p]
        lib.gm1b_flat_scalar_turbulence.restype = i32
        lib._turbs_bound = True
    return _launch(a, lib.gm1b_flat_scalar_turbulence, (ni, nj, nk, numq, ctypes.byref(s), dx, dy, dz, dt),
                   "gm1b_flat_scalar_turbulence",
                   {"stream": stream, "receipt": {"operator": "flat-scalar-turbulence", "scalars": 1 + numq,
                                                  "cell_words": ni * nj * nk}})


# ------------------------------------------------------ dissipative heating

DISSIPATIVE_HEATING_ARRAY_NAMES = ("dissten", "pi0", "ppi", "qa", "thten1")


class _DissArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in DISSIPATIVE_HEATING_ARRAY_NAMES]


def launch_cuda_dissipative_heating(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int,
                                    stream: Any | None = None) -> CudaLaunch:
    """CM1's dissipative heating (idiss = 1, Eqtset2IdissConsumer.apply,
    src/cm1core/eqtset2_energy_terms.py:375) added into ``thten1``:
    dissten (nk+1, nj, ni), pi0 (nk), ppi (nk, nj, ni), qa (6, nk, nj, ni)."""
    for name, value in (("ni", ni), ("nj", nj), ("nk", nk)):
        if isinstance(value, bool) or not isinstance(value, int) or value < 1:
            raise ValueError(f"{name} must be a positive integer")
    cell = (nk, nj, ni)
    shapes = {"dissten": (nk + 1, nj, ni), "pi0": (nk,), "ppi": cell, "qa": (6, nk, nj, ni), "thten1": cell}
    a = _require(arrays, DISSIPATIVE_HEATING_ARRAY_NAMES, shapes, "dissipative-heating")
    s = _DissArrays(**{n: a[n].data_ptr() for n in DISSIPATIVE_HEATING_ARRAY_NAMES})
    lib = _native.lib()
    if not getattr(lib, "_diss_bound", False):
        i32 = ctypes.c_int32
        lib.gm1b_dissipative_heating.argtypes = [i32, i32, i32, ctypes.POINTER(_DissArrays), ctypes.c_void_p]
        lib.gm1b_dissipative_heating.restype = i32
        lib._diss_bound = True
    return _launch(a, lib.gm1b_dissipative_heating, (ni, nj, nk, ctypes.byref(s)), "gm1b_dissipative_heating",
                   {"stream": stream, "receipt": {"operator": "dissipative-heating", "cell_words": ni * nj * nk}})


# ------------------------------------------------------- the terrain texts
# The uniform column's family: the strain of cpu_terrain_deformation_inplace
# (src/cm1core/cuda_terrain_deformation.py:234-736), gettau and turbu/turbv/
# turbw of cpu_sgs_stress_tendency_inplace
# (src/cm1core/cuda_sgs_stress_tendency.py:292-449), turbs of
# cpu_gm1_scalar_turbulence_inplace
# (src/cm1core/cuda_gm1_scalar_turbulence.py:230-430) - kernels in
# csrc/stress_terrain.cu.

TERRAIN_METRIC_NAMES = ("gz", "rgz", "gzu", "rgzu", "gzv", "rgzv", "gx", "gy", "gxu", "gyv")
_TERRAIN_FIELDS = ("u3d", "v3d", "w3d", "rho", "rf", "mh", "mf", "kmh", "kmv") + TERRAIN_METRIC_NAMES + \
    STRAIN_NAMES + TAU_NAMES + ("uten", "vten", "wten")
TERRAIN_STRAIN_ARRAY_NAMES = ("u3d", "v3d", "w3d", "rho", "rf", "gz", "rgz", "rgzu", "rgzv", "gx", "gy") + \
    STRAIN_NAMES
TERRAIN_STRESS_ARRAY_NAMES = STRAIN_NAMES + TAU_NAMES + ("kmh", "kmv", "rho", "rf", "mh", "mf", "gz", "rgz", "gzu",
                                                         "rgzu", "gzv", "rgzv", "gxu", "gyv", "u3d", "v3d", "w3d",
                                                         "uten", "vten", "wten")
TERRAIN_SGS_STRESS_ARRAY_NAMES = tuple(dict.fromkeys(TERRAIN_STRAIN_ARRAY_NAMES + TERRAIN_STRESS_ARRAY_NAMES))
TERRAIN_SCALAR_TURBULENCE_ARRAY_NAMES = ("th0", "tha", "qa", "rho", "rr", "rf", "mh", "mf", "khh", "khv", "gz",
                                         "rgz", "rgzu", "rgzv", "gx", "gxu", "gy", "gyv", "thten1", "qten",
                                         "workspace")


class _TerrainArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in _TERRAIN_FIELDS]


class _TerrainTurbsArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("th0", "tha", "qa", "rho", "rr", "rf", "mh", "mf", "khh", "khv",
                                               "gz", "rgz", "rgzu", "rgzv", "gx", "gxu", "gy", "gyv", "thten",
                                               "qten", "workspace")]


def terrain_metric_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    face = (nk + 1, nj, ni)
    return {"gz": (nj, ni), "rgz": (nj, ni), "gzu": (nj, ni + 1), "rgzu": (nj, ni + 1), "gzv": (nj + 1, ni),
            "rgzv": (nj + 1, ni), "gx": face, "gy": face, "gxu": (nk + 1, nj, ni + 1), "gyv": (nk + 1, nj + 1, ni)}


def terrain_stress_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    shapes = {n: s for n, s in flat_stress_shapes(ni, nj, nk).items() if n != "mh_profile"}
    shapes.update(terrain_metric_shapes(ni, nj, nk))
    return shapes


def _bind_terrain(lib) -> None:
    if getattr(lib, "_terrain_stress_bound", False):
        return
    i32, f32, vp = ctypes.c_int32, ctypes.c_float, ctypes.c_void_p
    a = ctypes.POINTER(_TerrainArrays)
    lib.gm1b_terrain_strain.argtypes = [i32, i32, i32, a, f32, f32, f32, vp]
    lib.gm1b_terrain_stress.argtypes = [i32, i32, i32, a, f32, f32, f32, f32, vp]
    lib.gm1b_terrain_sgs_stress.argtypes = [i32, i32, i32, a, f32, f32, f32, f32, vp]
    lib.gm1b_terrain_scalar_turbulence.argtypes = [i32, i32, i32, i32, ctypes.POINTER(_TerrainTurbsArrays), f32, f32,
                                                   f32, f32, vp]
    lib.gm1b_terrain_scalar_turbulence_workspace_words.argtypes = [i32, i32, i32, i32]
    lib.gm1b_terrain_scalar_turbulence_workspace_words.restype = ctypes.c_int64
    for n in ("gm1b_terrain_strain", "gm1b_terrain_stress", "gm1b_terrain_sgs_stress",
              "gm1b_terrain_scalar_turbulence"):
        getattr(lib, n).restype = i32
    lib._terrain_stress_bound = True


def _prepare_terrain(arrays: Mapping[str, Any], names, ni, nj, nk, what):
    _grid(ni, nj, nk)
    if nk > MAX_NK:
        raise ValueError(f"nk must be <= {MAX_NK} (the column solves' shared memory)")
    a = _require(arrays, names, terrain_stress_shapes(ni, nj, nk), what)
    s = _TerrainArrays(**{n: (a[n].data_ptr() if n in a else None) for n in _TERRAIN_FIELDS})
    lib = _native.lib()
    _bind_terrain(lib)
    return a, s, lib


def launch_cuda_terrain_strain(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float,
                               dz: float, stream: Any | None = None) -> CudaLaunch:
    """The strain carriers rho*Sij of the terrain calcdef: s11/s22/s33 at
    cells, s12 at every corner, s13/s23 on face levels 1..nk-1."""
    dx, dy, dz = _positive("dx", dx), _positive("dy", dy), _positive("dz", dz)
    a, s, lib = _prepare_terrain(arrays, TERRAIN_STRAIN_ARRAY_NAMES, ni, nj, nk, "terrain-strain")
    return _launch(a, lib.gm1b_terrain_strain, (ni, nj, nk, ctypes.byref(s), dx, dy, dz), "gm1b_terrain_strain",
                   {"stream": stream, "receipt": {"operator": "terrain-strain"}})


def launch_cuda_terrain_stress(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float,
                               dz: float, dt: float, stream: Any | None = None) -> CudaLaunch:
    """gettau and turbu/turbv/turbw of the terrain texts (four open sides,
    implicit vertical solves, free-slip bottom and top), the stress ADDED
    into uten/vten/wten (wten on faces 1..nk-1)."""
    dx, dy, dz, dt = _positive("dx", dx), _positive("dy", dy), _positive("dz", dz), _positive("dt", dt)
    a, s, lib = _prepare_terrain(arrays, TERRAIN_STRESS_ARRAY_NAMES, ni, nj, nk, "terrain-stress")
    return _launch(a, lib.gm1b_terrain_stress, (ni, nj, nk, ctypes.byref(s), dx, dy, dz, dt), "gm1b_terrain_stress",
                   {"stream": stream, "receipt": {"operator": "terrain-stress"}})


def launch_cuda_terrain_sgs_stress(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float,
                                   dz: float, dt: float, stream: Any | None = None) -> CudaLaunch:
    """The terrain strain carriers, gettau and the momentum stress in that
    order (cpu_sgs_stress_tendency_inplace with the strain its calcdef
    left)."""
    dx, dy, dz, dt = _positive("dx", dx), _positive("dy", dy), _positive("dz", dz), _positive("dt", dt)
    a, s, lib = _prepare_terrain(arrays, TERRAIN_SGS_STRESS_ARRAY_NAMES, ni, nj, nk, "terrain-sgs-stress")
    return _launch(a, lib.gm1b_terrain_sgs_stress, (ni, nj, nk, ctypes.byref(s), dx, dy, dz, dt),
                   "gm1b_terrain_sgs_stress", {"stream": stream, "receipt": {"operator": "terrain-sgs-stress"}})


def terrain_scalar_turbulence_workspace(ni: int, nj: int, nk: int, numq: int, device) -> torch.Tensor:
    """The device scratch launch_cuda_terrain_scalar_turbulence takes as
    ``workspace``: the x and y fluxes of each of the 1 + numq scalars."""
    return torch.empty((numq + 1) * (nk * nj * (ni + 1) + nk * (nj + 1) * ni), dtype=torch.float32, device=device)


def launch_cuda_terrain_scalar_turbulence(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, numq: int,
                                          dx: float, dy: float, dz: float, dt: float,
                                          stream: Any | None = None) -> CudaLaunch:
    """turbs on the terrain texts: theta ((th0 - 300) + tha) into
    ``thten1``, then moisture rows 0..numq-1 of ``qa`` into those of
    ``qten`` (added); the x/y fluxes with their terrain terms, the implicit
    vertical diffusion with khv, zero surface flux.  ``qa``/``qten`` may
    hold more rows than numq; ``workspace`` is
    terrain_scalar_turbulence_workspace()'s scratch."""
    if isinstance(numq, bool) or not isinstance(numq, int) or not 0 <= numq <= 6:
        raise ValueError("numq must be an integer in 0..6")
    dx, dy, dz, dt = _positive("dx", dx), _positive("dy", dy), _positive("dz", dz), _positive("dt", dt)
    _grid(ni, nj, nk)
    if nk > MAX_NK:
        raise ValueError(f"nk must be <= {MAX_NK} (the column solve's shared memory)")
    shapes = {n: s for n, s in flat_scalar_turbulence_shapes(ni, nj, nk, numq).items()}
    shapes.update(terrain_metric_shapes(ni, nj, nk))
    shapes["workspace"] = ((numq + 1) * (nk * nj * (ni + 1) + nk * (nj + 1) * ni),)
    for n in ("qa", "qten"):
        t = arrays.get(n)
        if isinstance(t, torch.Tensor) and t.dim() == 4 and t.shape[0] >= numq:
            shapes[n] = tuple(t.shape)
    a = _require(arrays, TERRAIN_SCALAR_TURBULENCE_ARRAY_NAMES, shapes, "terrain-scalar-turbulence")
    if tuple(a["qa"].shape[1:]) != (nk, nj, ni) or tuple(a["qten"].shape[1:]) != (nk, nj, ni):
        raise ValueError("qa and qten must hold rows of shape (nk, nj, ni)")
    s = _TerrainTurbsArrays(**{f: a["thten1" if f == "thten" else f].data_ptr()
                               for f, _ in _TerrainTurbsArrays._fields_})
    lib = _native.lib()
    _bind_terrain(lib)
    return _launch(a, lib.gm1b_terrain_scalar_turbulence, (ni, nj, nk, numq, ctypes.byref(s), dx, dy, dz, dt),
                   "gm1b_terrain_scalar_turbulence",
                   {"stream": stream, "receipt": {"operator": "terrain-scalar-turbulence", "scalars": 1 + numq,
                                                  "cell_words": ni * nj * nk}})
