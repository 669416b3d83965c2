"""CM1 vertical coordinates (stretch_z = 0 and 1) through libgm1b.so.

Mirrors (reference file:line):
  StretchZ1Parameters / StretchZ1Derived / derive_stretch_z1
      src/cm1core/cuda_stretch_z1.py:65-201
  launch_cuda_stretch_z1 -> CudaStretchZ1Launch(ready_event, grid, receipt)
      src/cm1core/cuda_stretch_z1.py:397-470
  VerticalLevels, build_vertical_levels, uniform_vertical_levels
      src/cm1core/cm1_vertical_grid.py:616-762, 780-937 (stretch_z 0 and 1)

Profiles are CM1-indexed float32: zf, sigmaf, mf, rmf, rdsf hold nk + 3
words, zh, sigma, mh, rmh, rds nk + 2.  ``build_vertical_levels`` forms them
on the host inside the library (as the reference's function does on the
host); ``launch_cuda_stretch_z1`` forms the same words on the device.
"""

from __future__ import annotations

import ctypes
import hashlib
from dataclasses import dataclass, field
from typing import Any

import numpy as np
import torch

from . import _native

PROFILES = ("zf", "zh", "sigmaf", "sigma", "mh", "mf", "rmh", "rmf", "rds", "rdsf")
LONG_PROFILES = ("zf", "sigmaf", "mf", "rmf", "rdsf")
ADMITTED_STRETCH_Z = (0, 1)
STRETCH_Z2_REFUSAL = ("stretch_z=2 is refused: CM1 r21.1 param.F:9897-9937 accepts whatever geometric ratio its "
                      "bisection holds, so its levels are not a function of the namelist words")
CUDA_STRETCH_Z1_SCHEMA = "gm1-b200.cuda-stretch-z1/v1"


class VerticalGridError(ValueError):
    """A vertical coordinate CM1 would stop on, or that is not built."""


@dataclass(frozen=True, slots=True)
class StretchZ1Parameters:
    nk: int
    dz: float
    ztop: float
    str_bot: float
    str_top: float
    dz_bot: float
    dz_top: float


@dataclass(frozen=True, slots=True)
class StretchZ1Derived:
    nk1: int
    nk2: int
    nk3: int
    nominal_dz_f32: float
    c1_f32: float
    c2_f32: float


class _Derived(ctypes.Structure):
    _fields_ = [("nk1", ctypes.c_int32), ("nk2", ctypes.c_int32), ("nk3", ctypes.c_int32),
                ("nominal", ctypes.c_float), ("c1", ctypes.c_float), ("c2", ctypes.c_float)]


class _Profiles(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in PROFILES]


def _lib():
    lib = _native.lib()
    if not getattr(lib, "_vertical_bound", False):
        f, i = ctypes.c_float, ctypes.c_int32
        lib.gm1b_stretch_z1_derive.argtypes = [i] + [f] * 6 + [ctypes.POINTER(_Derived)]
        lib.gm1b_vertical_levels.argtypes = [i, i] + [f] * 6 + [ctypes.POINTER(_Profiles),
                                                                ctypes.POINTER(ctypes.c_float),
                                                                ctypes.POINTER(ctypes.c_float)]
        lib.gm1b_stretch_z1.argtypes = [i] + [f] * 6 + [ctypes.POINTER(_Profiles), ctypes.c_void_p]
        for n in ("gm1b_stretch_z1_derive", "gm1b_vertical_levels", "gm1b_stretch_z1"):
            getattr(lib, n).restype = i
        lib._vertical_bound = True
    return lib


def _check(rc: int, what: str, error=VerticalGridError) -> None:
    if rc != 0:
        message = _native.lib().gm1b_last_error().decode("utf-8", errors="replace")
        raise error(f"{what}: {message}")


def _param_words(p: StretchZ1Parameters) -> list[float]:
    return [float(np.float32(v)) for v in (p.dz, p.ztop, p.str_bot, p.str_top, p.dz_bot, p.dz_top)]


def derive_stretch_z1(parameters: StretchZ1Parameters) -> StretchZ1Derived:
    """Segment counts and quadratic coefficients of a stretch_z = 1 column;
    ValueError on the reference's feasibility refusals."""
    if isinstance(parameters.nk, bool) or not isinstance(parameters.nk, int) or parameters.nk < 4:
        raise ValueError("nk must be an integer >= 4")
    d = _Derived()
    _check(_lib().gm1b_stretch_z1_derive(parameters.nk, *_param_words(parameters), ctypes.byref(d)),
           "derive_stretch_z1", ValueError)
    return StretchZ1Derived(d.nk1, d.nk2, d.nk3, float(d.nominal), float(d.c1), float(d.c2))


def _seal(arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float32).astype("<f4", copy=False).tobytes())
    return h.hexdigest()


@dataclass(frozen=True, eq=False)
class VerticalLevels:
    """One CM1 vertical coordinate, CM1-indexed and float32-exact."""

    stretch_z: int
    nk: int
    dz_reference_m: float
    ztop_m: float
    str_bot_m: float
    str_top_m: float
    dz_bot_m: float
    dz_top_m: float
    zf: np.ndarray
    zh: np.ndarray
    sigmaf: np.ndarray
    sigma: np.ndarray
    mh: np.ndarray
    mf: np.ndarray
    rmh: np.ndarray
    rmf: np.ndarray
    rds: np.ndarray
    rdsf: np.ndarray
    cgs: tuple[float, float, float]
    cgt: tuple[float, float, float]
    sha256: str = field(default="")

    @property
    def uniform(self) -> bool:
        return self.stretch_z == 0

    @property
    def mass_heights_m(self) -> tuple[float, ...]:
        return tuple(float(self.zh[k]) for k in range(1, self.nk + 1))

    @property
    def face_heights_m(self) -> tuple[float, ...]:
        return tuple(float(self.zf[k]) for k in range(1, self.nk + 2))

    @property
    def spacings_m(self) -> tuple[float, ...]:
        return tuple(float(self.zf[k + 1]) - float(self.zf[k]) for k in range(1, self.nk + 1))

    def stretch_parameters(self) -> StretchZ1Parameters:
        """The StretchZ1Parameters the device generator reproduces this column from."""
        if self.stretch_z == 0:
            return StretchZ1Parameters(self.nk, self.dz_reference_m, self.ztop_m, 0.0, self.ztop_m,
                                       self.dz_reference_m, self.dz_reference_m)
        return StretchZ1Parameters(self.nk, self.dz_reference_m, self.ztop_m, self.str_bot_m, self.str_top_m,
                                   self.dz_bot_m, self.dz_top_m)


def build_vertical_levels(*, stretch_z: int, nk: int, dz_m: float, ztop_m: float, str_bot_m: float = 0.0,
                          str_top_m: float = 0.0, dz_bot_m: float = 0.0, dz_top_m: float = 0.0,
                          levels_m=()) -> VerticalLevels:
    """One CM1 vertical coordinate for stretch_z 0 (param.F:7789-7811, top
    fixed at dz*nk) or 1 (Wilhelmson-Chen, param.F:7814-7953).  stretch_z 2
    is refused as the reference refuses it; the explicit-level branches 3 and
    4 are not built."""
    if isinstance(stretch_z, bool) or not isinstance(stretch_z, int):
        raise VerticalGridError("stretch_z must be an integer")
    if stretch_z == 2:
        raise VerticalGridError(STRETCH_Z2_REFUSAL)
    if stretch_z not in ADMITTED_STRETCH_Z:
        raise VerticalGridError(f"stretch_z={stretch_z} is not built here (stretch_z 0 and 1 are)")
    if isinstance(nk, bool) or not isinstance(nk, int) or nk < 4:
        raise VerticalGridError("nk must be an integer >= 4")
    if levels_m:
        raise VerticalGridError(f"stretch_z={stretch_z} carries no explicit levels")
    for name, v in (("dz_m", dz_m), ("ztop_m", ztop_m)):
        if isinstance(v, bool) or not isinstance(v, (int, float)) or not np.isfinite(v) or v <= 0:
            raise VerticalGridError(f"{name} must be finite and greater than zero")
    out = {n: np.zeros(nk + 3 if n in LONG_PROFILES else nk + 2, np.float32) for n in PROFILES}
    prof = _Profiles(**{n: out[n].ctypes.data for n in PROFILES})
    cgs = (ctypes.c_float * 3)()
    cgt = (ctypes.c_float * 3)()
    words = [float(np.float32(v)) for v in (dz_m, ztop_m, str_bot_m, str_top_m, dz_bot_m, dz_top_m)]
    _check(_lib().gm1b_vertical_levels(stretch_z, nk, *words, ctypes.byref(prof), cgs, cgt), "build_vertical_levels")
    for a in out.values():
        a.flags.writeable = False
    dz32 = float(np.float32(dz_m))
    if stretch_z == 0:
        top = float(np.float32(np.float32(dz_m) * np.float32(nk)))
        sb, st, db, dt = 0.0, top, dz32, dz32
    else:
        top = float(np.float32(ztop_m))
        sb, st, db, dt = (float(np.float32(v)) for v in (str_bot_m, str_top_m, dz_bot_m, dz_top_m))
    seal = _seal([out[n] for n in ("zf", "zh", "sigmaf", "sigma", "mh", "mf", "rmh", "rmf", "rds", "rdsf")])
    return VerticalLevels(stretch_z, nk, dz32, top, sb, st, db, dt, *(out[n] for n in PROFILES),
                          cgs=tuple(float(v) for v in cgs), cgt=tuple(float(v) for v in cgt), sha256=seal)


def uniform_vertical_levels(nk: int, dz_m: float) -> VerticalLevels:
    top = float(np.float32(np.float32(dz_m) * np.float32(nk)))
    return build_vertical_levels(stretch_z=0, nk=nk, dz_m=dz_m, ztop_m=top)


@dataclass(frozen=True, slots=True)
class DeviceStretchZ1Grid:
    zf: Any
    zh: Any
    sigmaf: Any
    sigma: Any
    mh: Any
    mf: Any
    rmh: Any
    rmf: Any
    rds: Any
    rdsf: Any
    derived: StretchZ1Derived


@dataclass(frozen=True, slots=True)
class CudaStretchZ1Launch:
    ready_event: Any
    grid: DeviceStretchZ1Grid
    receipt: dict[str, Any]


def launch_cuda_stretch_z1(parameters: StretchZ1Parameters, *, device: torch.device | str | None = None,
                           stream: Any | None = None) -> CudaStretchZ1Launch:
    """The stretch_z = 1 profiles (and rds/rdsf) as float32 CUDA tensors,
    formed on the device on ``stream``; ready_event records their completion."""
    derived = derive_stretch_z1(parameters)
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    st = torch.cuda.current_stream(dev) if stream is None else stream
    nk = parameters.nk
    with torch.cuda.stream(st):
        arrays = {n: torch.empty(nk + 3 if n in LONG_PROFILES else nk + 2, dtype=torch.float32, device=dev)
                  for n in PROFILES}
    prof = _Profiles(**{n: arrays[n].data_ptr() for n in PROFILES})
    _check(_lib().gm1b_stretch_z1(nk, *_param_words(parameters), ctypes.byref(prof), ctypes.c_void_p(st.cuda_stream)),
           "launch_cuda_stretch_z1")
    event = torch.cuda.Event()
    event.record(st)
    grid = DeviceStretchZ1Grid(*(arrays[n] for n in PROFILES), derived=derived)
    receipt = {"schema": CUDA_STRETCH_Z1_SCHEMA,
               "parameters": {n: getattr(parameters, n) for n in parameters.__dataclass_fields__},
               "derived": {n: getattr(derived, n) for n in derived.__dataclass_fields__}}
    return CudaStretchZ1Launch(event, grid, receipt)
