"""Kessler warm rain with saturation adjustment on B200.

Drop-in mirror of the reference operator API (torch CUDA tensors in place of
CuPy arrays; the same array names, shapes, dtypes, keywords and refusals):

  Gm1KesslerDriverSelection                 src/cm1core/cuda_gm1_kessler_driver.py:100-160
  gm1_kessler_driver_shapes                 src/cm1core/cuda_gm1_kessler_driver.py:183-206
  create_cuda_gm1_kessler_driver_workspace  src/cm1core/cuda_gm1_kessler_driver.py:806
  launch_cuda_gm1_kessler_driver            src/cm1core/cuda_gm1_kessler_driver.py:907
  launch_cuda_apmasscon, cpu_initial_dry_mass  src/cm1core/cuda_apmasscon.py:596, :226

Only efall = 0 is built (the benchmark configurations use it); efall = 1 is
refused by name.  Device faults never stand in for errors: the saturation
adjustment's non-convergence is a status word that ``CudaKesslerLaunch.check``
turns into the reference's RuntimeError.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Any, Mapping

import torch

from . import _native
from .errors import refuse


@dataclass(frozen=True, slots=True)
class Gm1KesslerDriverSelection:
    ptype: int = 1
    equation_set: int = 1
    testcase: int = 0
    pdscheme: int = 1
    efall: int = 0
    axisymmetric: int = 0
    moving_domain: int = 0
    rain_bins: int = 1
    nrk: int = 4
    input_phase: str = "pre-pdefq"
    output_phase: str = "post-satadj"


DEFAULT_GM1_KESSLER_DRIVER_SELECTION = Gm1KesslerDriverSelection()

INPUT_NAMES = ("ruh", "rvh", "rmh", "mh", "pi0", "th0", "rr")
INOUT_NAMES = ("rho", "pp3d", "th3d", "prs", "qv", "qc", "qr", "fall_velocity", "rain", "prate", "asq", "qbudget")
ALL_ARRAY_NAMES = INPUT_NAMES + INOUT_NAMES
DOUBLE_NAMES = ("asq", "qbudget")


def _validate_selection(selection: Gm1KesslerDriverSelection) -> None:
    if not isinstance(selection, Gm1KesslerDriverSelection):
        raise TypeError("selection must be a Gm1KesslerDriverSelection")
    fixed = {"ptype": 1, "testcase": 0, "pdscheme": 1, "axisymmetric": 0, "moving_domain": 0, "rain_bins": 1,
             "nrk": 4, "input_phase": "pre-pdefq", "output_phase": "post-satadj"}
    for name, wanted in fixed.items():
        value = getattr(selection, name)
        if type(value) is not type(wanted) or value != wanted:
            refuse(code="GM1-KESSLER-DRIVER-SELECTION", gate="physics-seam", option=name, value=value,
                   reason="the Kessler operator is built for one exact native branch",
                   remedy=f"use {name}={wanted!r}")
    if type(selection.efall) is not int or selection.efall != 0:
        refuse(code="GM1-KESSLER-DRIVER-EFALL", gate="physics-seam", option="efall", value=selection.efall,
               reason="only the disabled precipitation-energy fallout branch (efall=0) is built here",
               remedy="use efall=0")
    if type(selection.equation_set) is not int or selection.equation_set not in (1, 2):
        refuse(code="GM1-KESSLER-DRIVER-EQTSET", gate="physics-seam", option="equation_set",
               value=selection.equation_set,
               reason="the authority has exactly traditional and energy-conserving branches",
               remedy="use equation_set=1 or equation_set=2")


def gm1_kessler_driver_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    for name, value in (("ni", ni), ("nj", nj), ("nk", nk)):
        if type(value) is not int or value < 1:
            raise ValueError(f"{name} must be an integer >= 1")
    mass = (nk, nj, ni)
    shapes = {name: mass for name in ("rmh", "mh", "pi0", "th0", "rho", "rr", "pp3d", "th3d", "prs", "qv", "qc",
                                      "qr", "fall_velocity")}
    shapes.update({"ruh": (ni,), "rvh": (nj,), "rain": (1, nj, ni), "prate": (nj, ni), "asq": (3,),
                   "qbudget": (10,)})
    return shapes


class _KesslerArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in (*INPUT_NAMES, "rho", "pp3d", "th3d", "prs", "qv", "qc", "qr",
                                               "fall_velocity", "rain", "prate", "asq", "qbudget",
                                               "satadj_iterations", "nfall")]


def _bind() -> ctypes.CDLL:
    lib = _native.lib()
    if not getattr(lib, "_kessler_bound", False):
        i32, f32 = ctypes.c_int32, ctypes.c_float
        lib.gm1b_kessler_workspace_bytes.argtypes = [i32, i32, i32]
        lib.gm1b_kessler_workspace_bytes.restype = ctypes.c_size_t
        lib.gm1b_kessler_driver.argtypes = [i32, i32, i32, ctypes.POINTER(_KesslerArrays), f32, f32, f32, f32, i32,
                                            i32, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        lib.gm1b_kessler_driver.restype = i32
        lib._kessler_bound = True
    return lib


@dataclass
class Gm1KesslerDriverWorkspace:
    """Caller-owned device scratch of the operator (budget partial sums and
    the two status words)."""

    ni: int
    nj: int
    nk: int
    buffer: torch.Tensor

    @property
    def status(self) -> torch.Tensor:
        return self.buffer[:16].view(torch.int32)


def create_cuda_gm1_kessler_driver_workspace(*, ni: int, nj: int, nk: int,
                                             device: torch.device | str = "cuda") -> Gm1KesslerDriverWorkspace:
    gm1_kessler_driver_shapes(ni, nj, nk)
    nbytes = int(_bind().gm1b_kessler_workspace_bytes(ni, nj, nk))
    buf = torch.empty(((nbytes + 255) // 256) * 256, dtype=torch.uint8, device=device)
    return Gm1KesslerDriverWorkspace(ni, nj, nk, buf)


@dataclass(frozen=True)
class CudaKesslerLaunch:
    ready_event: torch.cuda.Event
    workspace: Gm1KesslerDriverWorkspace
    receipt: dict[str, Any]

    def status(self) -> dict[str, int]:
        """Waits for the launch and reads its status words."""
        self.ready_event.synchronize()
        s = self.workspace.status.cpu().tolist()
        return {"satadj_nonconverged_cells": int(s[0]), "max_fall_substeps": int(s[1]),
                "blown_up_fall_columns": int(s[2])}

    def check(self) -> dict[str, int]:
        """status(), raising like the reference if any saturation adjustment
        did not converge within 100 iterations, and if a rain column's fall
        Courant number was not finite or reached 16384 (a blown-up state that
        the operator stepped once instead of int(crmax + 1) times)."""
        s = self.status()
        if s["satadj_nonconverged_cells"]:
            raise RuntimeError("GM1 Kessler satadj failed to converge in 100 iterations "
                               f"({s['satadj_nonconverged_cells']} cells)")
        if s["blown_up_fall_columns"]:
            raise RuntimeError(f"GM1 Kessler fallout: {s['blown_up_fall_columns']} columns with a fall Courant "
                               "number that is not finite or at least 16384")
        return s


def _positive(name: str, value: float) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise TypeError(f"{name} must be a finite positive number")
    result = float(value)
    if not math.isfinite(result) or result <= 0.0:
        raise ValueError(f"{name} must be finite and > 0")
    return result


def launch_cuda_gm1_kessler_driver(
    arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float, dz: float, dt: float,
    selection: Gm1KesslerDriverSelection = DEFAULT_GM1_KESSLER_DRIVER_SELECTION, stream: Any | None = None,
    workspace: Gm1KesslerDriverWorkspace | None = None, satadj_iterations: torch.Tensor | None = None,
    nfall: torch.Tensor | None = None,
) -> CudaKesslerLaunch:
    """Enqueue the complete Kessler operator in place without synchronising."""
    _validate_selection(selection)
    shapes = gm1_kessler_driver_shapes(ni, nj, nk)
    dx, dy, dz, dt = (_positive(n, v) for n, v in (("dx", dx), ("dy", dy), ("dz", dz), ("dt", dt)))
    missing = [n for n in ALL_ARRAY_NAMES if n not in arrays]
    if missing:
        raise ValueError(f"missing GM1 Kessler driver arrays: {', '.join(missing)}")
    a: dict[str, torch.Tensor] = {}
    for n in ALL_ARRAY_NAMES:
        t = arrays[n]
        dtype = torch.float64 if n in DOUBLE_NAMES else torch.float32
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != dtype or tuple(t.shape) != shapes[n] \
                or not t.is_contiguous():
            raise ValueError(f"{n} must be a contiguous CUDA {dtype} tensor with shape {shapes[n]}")
        a[n] = t
    if satadj_iterations is not None:
        if satadj_iterations.dtype != torch.int32 or tuple(satadj_iterations.shape) != (nk, nj, ni):
            raise ValueError("satadj_iterations must be an int32 (uint32 words) tensor of the mass shape")
        a["satadj_iterations"] = satadj_iterations
    if nfall is not None:
        if nfall.dtype != torch.int32 or tuple(nfall.shape) != (nj, ni):
            raise ValueError("nfall must be an int32 tensor of shape (nj, ni)")
        a["nfall"] = nfall
    ptrs = [t.data_ptr() for t in a.values()]
    if len(set(ptrs)) != len(ptrs):
        raise ValueError("GM1 Kessler driver arrays must not alias")
    device = a["rho"].device
    if workspace is None:
        workspace = create_cuda_gm1_kessler_driver_workspace(ni=ni, nj=nj, nk=nk, device=device)
    elif (workspace.ni, workspace.nj, workspace.nk) != (ni, nj, nk):
        raise ValueError("workspace was created for another grid")
    s = _KesslerArrays(**{n: t.data_ptr() for n, t in a.items()})
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        _native.check(_bind().gm1b_kessler_driver(ni, nj, nk, ctypes.byref(s), dx, dy, dz, dt,
                                                  selection.equation_set, selection.efall,
                                                  ctypes.c_void_p(workspace.buffer.data_ptr()),
                                                  workspace.buffer.numel(), ctypes.c_void_p(st.cuda_stream)),
                      "gm1b_kessler_driver")
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaKesslerLaunch(ev, workspace, {"operator": "gm1-kessler-driver", "equation_set": selection.equation_set,
                                             "efall": selection.efall, "domain": {"ni": ni, "nj": nj, "nk": nk}})


# ---------------------------------------------------------------------------
# once-per-large-step transition (src/cm1core/cuda_gm1_kessler_large_step.py)
# ---------------------------------------------------------------------------
HELD_NAMES = ("qpten", "qtten", "qvten", "qcten")


@dataclass(slots=True)
class Gm1KesslerHeldCarriers:
    qpten: torch.Tensor
    qtten: torch.Tensor
    qvten: torch.Tensor
    qcten: torch.Tensor


class _HeldArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in HELD_NAMES]


@dataclass(frozen=True, slots=True)
class Gm1KesslerLargeStepResult:
    ready_event: Any
    completed_transitions: int
    receipt: Mapping[str, Any]


class CudaGm1KesslerLargeStepTransition:
    """Persistent source-ordered Kessler transition of one CUDA state: held
    rate remove/snapshot, pre-physics EOS, the driver, held recapture, all in
    one library call (gm1b_kessler_large_step)."""

    def __init__(self, arrays: dict[str, torch.Tensor], carriers: Gm1KesslerHeldCarriers, *, ni: int, nj: int,
                 nk: int, dx: float, dy: float, dz: float, dt: float, selection: Gm1KesslerDriverSelection,
                 stream: Any, workspace: Gm1KesslerDriverWorkspace, completed_transitions: int = 0,
                 mass1: torch.Tensor | None = None) -> None:
        self.arrays, self.carriers = arrays, carriers
        self.ni, self.nj, self.nk = ni, nj, nk
        self.dx, self.dy, self.dz, self.dt = dx, dy, dz, dt
        self.selection, self.stream, self.workspace = selection, stream, workspace
        self.completed_transitions = completed_transitions
        # with a dry-mass ledger: the final-RK dry-air mass correction between
        # the pre-physics equation of state and the driver (the reference's
        # dry-mass hook at that point, CM1 apmasscon = 1)
        self.mass1 = mass1
        self.mass_workspace = None if mass1 is None else torch.empty(
            (_apmasscon_lib().gm1b_apmasscon_workspace_bytes(nk) + 7) // 8, dtype=torch.float64, device=mass1.device)
        self.mass_diagnostics = None if mass1 is None else torch.zeros(4, dtype=torch.float64, device=mass1.device)

    def apply(self, *, final_rk: bool = True, refl_10cm_due: bool = False,
              pre_component_hook: Any | None = None) -> Gm1KesslerLargeStepResult:
        if type(final_rk) is not bool or not final_rk:
            refuse(code="GM1-KESSLER-LARGE-STEP-CADENCE", gate="physics-seam", option="final_rk", value=final_rk,
                   reason="CM1 r21.1 calls mp_driver once after the completed RK solve",
                   remedy="invoke the transition only after final RK stage 3")
        if type(refl_10cm_due) is not bool:
            raise TypeError("refl_10cm_due must be boolean")
        if refl_10cm_due:
            refuse(code="GM1-KESSLER-REFLECTIVITY-UNPORTED", gate="physics-seam", option="refl_10cm_due",
                   value=True, reason="CM1 does not admit the selected reflectivity consumer for ptype=1",
                   remedy="disable reflectivity or select an admitted microphysics consumer")
        if pre_component_hook is not None:
            refuse(code="GM1-KESSLER-LARGE-STEP-HOOK", gate="physics-seam", option="pre_component_hook",
                   value=type(pre_component_hook).__name__,
                   reason="the dry-mass hook between the pre-physics EOS and the driver is not part of this "
                          "operator (one fused library call)", remedy="run the transition without a hook")
        a, h = self.arrays, self.carriers
        s = _KesslerArrays(**{n: t.data_ptr() for n, t in a.items() if n in ALL_ARRAY_NAMES})
        held = _HeldArrays(**{n: getattr(h, n).data_ptr() for n in HELD_NAMES})
        device = a["rho"].device
        st = torch.cuda.current_stream(device) if self.stream is None else self.stream
        lib = _bind()
        if not getattr(lib, "_kls_bound", False):
            c = ctypes
            lib.gm1b_kessler_large_step.argtypes = [c.c_int32] * 3 + [c.POINTER(_KesslerArrays), c.POINTER(_HeldArrays)] + \
                [c.c_float] * 4 + [c.c_int32, c.c_int32, c.c_void_p, c.c_size_t, c.c_void_p]
            lib.gm1b_kessler_large_step.restype = c.c_int32
            lib._kls_bound = True
        with torch.cuda.device(device):
            if self.mass1 is None:
                _native.check(lib.gm1b_kessler_large_step(
                    self.ni, self.nj, self.nk, ctypes.byref(s), ctypes.byref(held), self.dx, self.dy, self.dz,
                    self.dt, self.selection.equation_set, self.selection.efall,
                    ctypes.c_void_p(self.workspace.buffer.data_ptr()), self.workspace.buffer.numel(),
                    ctypes.c_void_p(st.cuda_stream)), "gm1b_kessler_large_step")
            else:
                _native.check(_apmasscon_lib().gm1b_kessler_large_step_apmasscon(
                    self.ni, self.nj, self.nk, ctypes.byref(s), ctypes.byref(held), self.dx, self.dy, self.dz,
                    self.dt, self.selection.equation_set, self.selection.efall,
                    ctypes.c_void_p(self.workspace.buffer.data_ptr()), self.workspace.buffer.numel(),
                    ctypes.c_void_p(self.mass1.data_ptr()), ctypes.c_void_p(self.mass_diagnostics.data_ptr()),
                    ctypes.c_void_p(self.mass_workspace.data_ptr()), ctypes.c_void_p(st.cuda_stream)),
                    "gm1b_kessler_large_step_apmasscon")
            ev = torch.cuda.Event()
            ev.record(st)
        self.completed_transitions += 1
        return self._result(ev)

    def _structs(self):
        a, h = self.arrays, self.carriers
        s = _KesslerArrays(**{n: t.data_ptr() for n, t in a.items() if n in ALL_ARRAY_NAMES})
        held = _HeldArrays(**{n: getattr(h, n).data_ptr() for n in HELD_NAMES})
        st = torch.cuda.current_stream(a["rho"].device) if self.stream is None else self.stream
        return s, held, st

    def begin(self, window: tuple[int, int, int, int], partials: torch.Tensor) -> None:
        """The transition of a subdomain up to the dry-mass ledger: held
        rates removed, the pre-physics EOS, and the level partials of its own
        cells (window = (i0, i1, j0, j1) columns and rows) into partials
        (float64, apmasscon_partials_words(nk) words)."""
        if self.mass1 is None:
            raise RuntimeError("begin/end split the dry-mass correction: build the transition with mass1")
        s, held, st = self._structs()
        w = (ctypes.c_int32 * 4)(*window)
        with torch.cuda.device(self.arrays["rho"].device):
            _native.check(_apmasscon_lib().gm1b_kessler_large_step_apmasscon_begin(
                self.ni, self.nj, self.nk, ctypes.byref(s), ctypes.byref(held), self.dt, self.selection.equation_set,
                w, ctypes.c_void_p(partials.data_ptr()), ctypes.c_void_p(st.cuda_stream)),
                "gm1b_kessler_large_step_apmasscon_begin")

    def end(self, partials: torch.Tensor, cells: int) -> Gm1KesslerLargeStepResult:
        """The rest of the transition from the domain's added partials: the
        correction for `cells` cells, the driver, the recapture."""
        s, held, st = self._structs()
        with torch.cuda.device(self.arrays["rho"].device):
            _native.check(_apmasscon_lib().gm1b_kessler_large_step_apmasscon_end(
                self.ni, self.nj, self.nk, ctypes.byref(s), ctypes.byref(held), self.dx, self.dy, self.dz, self.dt,
                self.selection.equation_set, self.selection.efall, ctypes.c_void_p(self.workspace.buffer.data_ptr()),
                self.workspace.buffer.numel(), ctypes.c_void_p(partials.data_ptr()), float(cells),
                ctypes.c_void_p(self.mass1.data_ptr()), ctypes.c_void_p(self.mass_diagnostics.data_ptr()),
                ctypes.c_void_p(self.mass_workspace.data_ptr()), ctypes.c_void_p(st.cuda_stream)),
                "gm1b_kessler_large_step_apmasscon_end")
            ev = torch.cuda.Event()
            ev.record(st)
        self.completed_transitions += 1
        return self._result(ev)

    def _result(self, ev) -> Gm1KesslerLargeStepResult:
        return Gm1KesslerLargeStepResult(ev, self.completed_transitions, {
            "operator": "gm1-kessler-large-step", "equation_set": self.selection.equation_set,
            "source_order": ("solve2-held-remove-snapshot", "solve2-pre-physics-eos") +
                            (() if self.mass1 is None else ("solve2-apmasscon",)) +
                            ("cm1-mp_driver-ptype1", "solve3-held-recapture"),
            "domain": {"ni": self.ni, "nj": self.nj, "nk": self.nk}})


def create_cuda_gm1_kessler_large_step_transition(
        arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, dx: float, dy: float, dz: float, dt: float,
        selection: Gm1KesslerDriverSelection, stream: Any | None = None,
        workspace: Gm1KesslerDriverWorkspace | None = None,
        carriers: Gm1KesslerHeldCarriers | None = None,
        mass1: torch.Tensor | None = None) -> CudaGm1KesslerLargeStepTransition:
    """Bind an already Kessler-initialised device state.  rr, fall_velocity,
    rain, prate, asq and qbudget are allocated (zero) when absent, as are the
    held carriers (the reference's fresh-start restart state)."""
    for name, value, minimum in (("ni", ni, 1), ("nj", nj, 1), ("nk", nk, 2)):
        if type(value) is not int or value < minimum:
            raise ValueError(f"{name} must be an integer >= {minimum}")
    dx, dy, dz, dt = (_positive(n, v) for n, v in (("dx", dx), ("dy", dy), ("dz", dz), ("dt", dt)))
    _validate_selection(selection)
    shapes = gm1_kessler_driver_shapes(ni, nj, nk)
    base = ("ruh", "rvh", "rmh", "mh", "pi0", "th0", "rho", "pp3d", "th3d", "prs", "qv", "qc", "qr")
    missing = [n for n in base if n not in arrays]
    if missing:
        raise ValueError("missing GM1 Kessler large-step arrays: " + ", ".join(missing))
    device = arrays["rho"].device
    bound: dict[str, torch.Tensor] = {}
    for n in ALL_ARRAY_NAMES:
        dtype = torch.float64 if n in DOUBLE_NAMES else torch.float32
        t = arrays.get(n)
        if t is None and n not in base:
            t = torch.zeros(shapes[n], dtype=dtype, device=device)
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != dtype or tuple(t.shape) != shapes[n] \
                or not t.is_contiguous():
            raise ValueError(f"{n} must be C-order CUDA {dtype} with shape {shapes[n]}")
        bound[n] = t
    if len({t.data_ptr() for t in bound.values()}) != len(bound):
        raise ValueError("GM1 Kessler large-step arrays must not alias")
    mass = (nk, nj, ni)
    if carriers is None:
        carriers = Gm1KesslerHeldCarriers(*(torch.zeros(mass, device=device) for _ in HELD_NAMES))
    for n in HELD_NAMES:
        t = getattr(carriers, n)
        if not isinstance(t, torch.Tensor) or t.dtype != torch.float32 or tuple(t.shape) != mass \
                or not t.is_contiguous() or t.device != device:
            raise ValueError(f"held {n} must be C-order CUDA float32 with shape {mass}")
    if workspace is None:
        workspace = create_cuda_gm1_kessler_driver_workspace(ni=ni, nj=nj, nk=nk, device=device)
    if mass1 is not None and (not isinstance(mass1, torch.Tensor) or mass1.dtype != torch.float64
                              or tuple(mass1.shape) != (1,) or mass1.device != device):
        raise ValueError("mass1 must be a one-word float64 tensor on the state's device")
    return CudaGm1KesslerLargeStepTransition(bound, carriers, ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, dz=dz, dt=dt,
                                             selection=selection, stream=stream, workspace=workspace, mass1=mass1)


# ---------------------------------------------------------------------------
# the final-RK dry-air mass correction (apmasscon = 1)
# ---------------------------------------------------------------------------
APMASSCON_INPUT_NAMES = ("ruh", "rvh", "rmh", "pi0", "th0", "th3d", "qv")
APMASSCON_MUTABLE_NAMES = ("pp3d", "prs", "rho")
APMASSCON_ARRAY_NAMES = APMASSCON_INPUT_NAMES + APMASSCON_MUTABLE_NAMES


class _ApMassConArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in APMASSCON_ARRAY_NAMES]


def _apmasscon_lib() -> ctypes.CDLL:
    lib = _native.lib()
    if not getattr(lib, "_apmasscon_bound", False):
        c = ctypes
        lib.gm1b_apmasscon_workspace_bytes.argtypes = [c.c_int32]
        lib.gm1b_apmasscon_workspace_bytes.restype = c.c_size_t
        lib.gm1b_apmasscon.argtypes = [c.c_int32] * 3 + [c.POINTER(_ApMassConArrays), c.c_void_p, c.c_void_p,
                                                         c.c_void_p, c.c_void_p]
        lib.gm1b_apmasscon.restype = c.c_int32
        lib.gm1b_dry_mass.argtypes = [c.c_int32] * 3 + [c.c_void_p] * 5 + [c.c_int32, c.c_void_p, c.c_void_p]
        lib.gm1b_dry_mass.restype = c.c_int32
        lib.gm1b_kessler_large_step_apmasscon.argtypes = [c.c_int32] * 3 + [c.POINTER(_KesslerArrays),
                                                                            c.POINTER(_HeldArrays)] + \
            [c.c_float] * 4 + [c.c_int32, c.c_int32, c.c_void_p, c.c_size_t] + [c.c_void_p] * 4
        lib.gm1b_kessler_large_step_apmasscon.restype = c.c_int32
        lib.gm1b_apmasscon_partials_words.argtypes = [c.c_int32]
        lib.gm1b_apmasscon_partials_words.restype = c.c_size_t
        lib.gm1b_apmasscon_partials.argtypes = [c.c_int32] * 3 + [c.c_void_p] * 6 + [c.POINTER(c.c_int32), c.c_int32,
                                                                                     c.c_void_p, c.c_void_p]
        lib.gm1b_apmasscon_partials.restype = c.c_int32
        lib.gm1b_dry_mass_from_partials.argtypes = [c.c_int32, c.c_void_p, c.c_void_p, c.c_int32, c.c_void_p]
        lib.gm1b_dry_mass_from_partials.restype = c.c_int32
        lib.gm1b_kessler_large_step_apmasscon_begin.argtypes = [c.c_int32] * 3 + [c.POINTER(_KesslerArrays),
                                                                                  c.POINTER(_HeldArrays), c.c_float,
                                                                                  c.c_int32, c.POINTER(c.c_int32),
                                                                                  c.c_void_p, c.c_void_p]
        lib.gm1b_kessler_large_step_apmasscon_begin.restype = c.c_int32
        lib.gm1b_kessler_large_step_apmasscon_end.argtypes = [c.c_int32] * 3 + [c.POINTER(_KesslerArrays),
                                                                                c.POINTER(_HeldArrays)] + \
            [c.c_float] * 4 + [c.c_int32, c.c_int32, c.c_void_p, c.c_size_t, c.c_void_p, c.c_double] + [c.c_void_p] * 4
        lib.gm1b_kessler_large_step_apmasscon_end.restype = c.c_int32
        lib._apmasscon_bound = True
    return lib


def apmasscon_partials_words(nk: int) -> int:
    return int(_apmasscon_lib().gm1b_apmasscon_partials_words(nk))


def dry_mass_partials(rho, ruh, rvh, rmh, *, ni: int, nj: int, nk: int, window: tuple[int, int, int, int],
                      partials: torch.Tensor, stream: Any | None = None) -> torch.Tensor:
    """The dry-mass ledger's level partials over a window of cells (a
    subdomain's own), to be added over the subdomains and finished by
    dry_mass_from_partials."""
    st = torch.cuda.current_stream(rho.device) if stream is None else stream
    w = (ctypes.c_int32 * 4)(*window)
    with torch.cuda.device(rho.device):
        _native.check(_apmasscon_lib().gm1b_apmasscon_partials(
            ni, nj, nk, rho.data_ptr(), ruh.data_ptr(), rvh.data_ptr(), rmh.data_ptr(), None, None, w, 0,
            partials.data_ptr(), ctypes.c_void_p(st.cuda_stream)), "gm1b_apmasscon_partials")
    return partials


def dry_mass_from_partials(partials: torch.Tensor, nk: int, out: torch.Tensor, stream: Any | None = None) -> None:
    st = torch.cuda.current_stream(out.device) if stream is None else stream
    with torch.cuda.device(out.device):
        _native.check(_apmasscon_lib().gm1b_dry_mass_from_partials(nk, partials.data_ptr(), out.data_ptr(), 0,
                                                                   ctypes.c_void_p(st.cuda_stream)),
                      "gm1b_dry_mass_from_partials")


def apmasscon_array_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    scalar = (nk, nj, ni)
    return {"ruh": (ni,), "rvh": (nj,), **{n: scalar for n in APMASSCON_ARRAY_NAMES if n not in ("ruh", "rvh")}}


def _mass_arrays(arrays: Mapping[str, Any], ni: int, nj: int, nk: int) -> dict[str, torch.Tensor]:
    shapes = apmasscon_array_shapes(ni, nj, nk)
    missing = [n for n in APMASSCON_ARRAY_NAMES if n not in arrays]
    if missing:
        raise ValueError(f"missing apmasscon arrays: {', '.join(missing)}")
    out = {}
    for n in APMASSCON_ARRAY_NAMES:
        t = arrays[n]
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 \
                or tuple(t.shape) != shapes[n] or not t.is_contiguous():
            raise ValueError(f"{n} must be C-order CUDA float32 with shape {shapes[n]}")
        out[n] = t
    if len({t.data_ptr() for t in out.values()}) != len(out):
        raise ValueError("apmasscon arrays must not alias")
    return out


def _mass_word(mass1: Any, device: torch.device) -> torch.Tensor:
    if isinstance(mass1, torch.Tensor):
        if mass1.dtype != torch.float64 or tuple(mass1.shape) != (1,) or mass1.device != device:
            raise ValueError("mass1 must be a one-word float64 tensor on the arrays' device")
        return mass1
    if isinstance(mass1, bool) or not isinstance(mass1, (int, float)) or not math.isfinite(mass1) or mass1 <= 0.0:
        raise ValueError("mass1 must be a finite positive dry-air mass")
    return torch.tensor([float(mass1)], dtype=torch.float64, device=device)


@dataclass(frozen=True, slots=True)
class CudaApMassConLaunch:
    ready_event: Any
    diagnostics: torch.Tensor  # mass2, Exner sum, binary64 correction, mass1
    receipt: Mapping[str, Any]


def launch_cuda_apmasscon(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int, mass1: Any,
                          stream: Any | None = None) -> CudaApMassConLaunch:
    """The final-RK dry-air mass correction in place (pp3d, prs, rho),
    without host synchronization; mass1 a float or a one-word float64 device
    tensor (the initial ledger)."""
    for name, value in (("ni", ni), ("nj", nj), ("nk", nk)):
        if type(value) is not int or value < 1:
            raise ValueError(f"{name} must be an integer >= 1")
    a = _mass_arrays(arrays, ni, nj, nk)
    device = a["rho"].device
    m1 = _mass_word(mass1, device)
    lib = _apmasscon_lib()
    work = torch.empty((lib.gm1b_apmasscon_workspace_bytes(nk) + 7) // 8, dtype=torch.float64, device=device)
    diag = torch.zeros(4, dtype=torch.float64, device=device)
    st = torch.cuda.current_stream(device) if stream is None else stream
    s = _ApMassConArrays(**{n: a[n].data_ptr() for n in APMASSCON_ARRAY_NAMES})
    with torch.cuda.device(device):
        _native.check(lib.gm1b_apmasscon(ni, nj, nk, ctypes.byref(s), m1.data_ptr(), diag.data_ptr(), work.data_ptr(),
                                         ctypes.c_void_p(st.cuda_stream)), "gm1b_apmasscon")
        for t in (work, m1, diag):  # temporaries in use on st until it reaches here
            t.record_stream(st)
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaApMassConLaunch(ev, diag, {"operator": "gm1-apmasscon", "domain": {"ni": ni, "nj": nj, "nk": nk},
                                          "source_order": ("layer-reductions", "correction", "eos-rebuild")})


def dry_mass(rho: torch.Tensor, ruh: torch.Tensor, rvh: torch.Tensor, rmh: torch.Tensor, *, ni: int, nj: int, nk: int,
             out: torch.Tensor | None = None, only_if_unset: bool = False, stream: Any | None = None) -> torch.Tensor:
    """The dry-air mass ledger of a state (cpu_initial_dry_mass) into a
    one-word float64 device tensor; with only_if_unset a non-zero out is kept."""
    device = rho.device
    for n, t, shape in (("rho", rho, (nk, nj, ni)), ("ruh", ruh, (ni,)), ("rvh", rvh, (nj,)), ("rmh", rmh, (nk, nj, ni))):
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 or tuple(t.shape) != shape \
                or not t.is_contiguous():
            raise ValueError(f"{n} must be C-order CUDA float32 with shape {shape}")
    if out is None:
        out = torch.zeros(1, dtype=torch.float64, device=device)
    lib = _apmasscon_lib()
    work = torch.empty((lib.gm1b_apmasscon_workspace_bytes(nk) + 7) // 8, dtype=torch.float64, device=device)
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        _native.check(lib.gm1b_dry_mass(ni, nj, nk, rho.data_ptr(), ruh.data_ptr(), rvh.data_ptr(), rmh.data_ptr(),
                                        out.data_ptr(), 1 if only_if_unset else 0, work.data_ptr(),
                                        ctypes.c_void_p(st.cuda_stream)), "gm1b_dry_mass")
        work.record_stream(st)
    return out
