"""The moist large step on B200: the operators of this package composed in
the reference's large-step schedule (StepPhase / large_step_schedule,
src/cm1core/gm1_runtime.py:611-627, :1969-2007) on the padded (ng = 3)
open-lateral lane with Kessler warm rain, WENO5 moisture and the 1.5-order
TKE closure.

Phase bindings (reference phase methods they follow):

  CLOSURE             calcnm, calcdef, tkekm + TKE source, turbt once per step
                      (CartesianClosure, src/cm1core/cuda_cartesian_closure.py:1118-1200)
  HELD_TENDENCIES     held theta/qv/qc rates and ppten (finalize_held_tendencies,
                      src/cm1core/cuda_cartesian_dynamics.py:1014)
  PRE_ACOUSTIC        eqtset2 stage terms, w(1) surface fill, momentum advection with the
                      bcw(rrw) lateral fill between mass flux and transport, moist buoyancy (:1047-1125)
  ACOUSTIC            terrain/open psolver3 stage without its stage fills (:1127-1202)
  POST_ACOUSTIC       getdiv on the averaged velocities, getdivx mass fluxes and divx (:1204-1233)
  SCALAR_MOIST        theta and qv/qc/qr advection (WENO5 at nrk = 3) and the RK update; the
                      final stage's moisture advection is the pdef chain alone (:1235-1274)
  MOMENTUM_BOUNDARIES bcu, bcv, bcw(flag 1), bcwsfc (:1276-1297)
  SCALAR_BOUNDARIES   bcp of pp3d between stages (:1299-1318)
  TKE                 TKE advection + RK stage (CartesianClosure.tke_rk, :1635)
  MICROPHYSICS        the Kessler once-per-large-step transition: held-rate remove and snapshot,
                      pre-physics EOS, the Kessler operator, held-rate recapture
                      (cpu_gm1_kessler_large_step_inplace, src/cm1core/cuda_gm1_kessler_large_step.py:183);
                      REMOVE_HELD_EOS and POST_PHYSICS are its first and last parts
  SOLVE3              ppx accumulation, A-level promotion, rr/rf (cuda_cartesian_finish.py:739)

Left out identically in this composition and in the oracle's: SGS stress and
scalar diffusion tendencies, Rayleigh damping, the dry-mass correction
(MASS_BEGIN / MASS_FINISH), surface fluxes.  Terrain metrics may be flat
(gz = 1, zero slopes); every operator keeps its terrain arithmetic.
"""

from __future__ import annotations

import ctypes
import functools
from dataclasses import dataclass
from enum import Enum
from typing import Any

import numpy as np
import torch

from . import _native
from . import moist_ops as mo
from .advection import launch_cuda_gm1_child_stretched_scalar_advection5, launch_cuda_scalar_advection5
from .closure import launch_cuda_flat_deformation, launch_cuda_moist_nm, launch_cuda_terrain_deformation
from .kessler import (Gm1KesslerDriverSelection, Gm1KesslerHeldCarriers, create_cuda_gm1_kessler_large_step_transition,
                      dry_mass)
from .errors import refuse
from .limits import CM1_COURANT_STOP, advective_courant_number
from .moist_bridge import launch_cuda_eqtset2_stage_terms
from .scalar_rk import (compose_scalar_moist_rk_stage, moisture_weps_f64, scalar_moist_rk_stage_timestep_f32,
                        theta_transport_scalar, theta_weps_f64)
from .terrain_open import (ALL_ARRAY_NAMES as TOS_ARRAY_NAMES, COLUMN_DIAGNOSTIC_NAMES, GM1B_TOS_DIAGNOSTICS,
                           _STRUCT_METRICS as TOS_METRICS, _Arrays as _TosArrays, _Metrics as _TosMetrics,
                           _lib as _tos_lib)
from .tke import launch_cuda_sgs_tke
from .tke_evolution import (launch_cuda_flat_tke_diffusion, launch_cuda_flat_tke_rk_stage, launch_cuda_tke_diffusion,
                            launch_cuda_tke_rk_stage)


class MoistStepFailure(RuntimeError):
    """A composed step reached a state the reference refuses to continue."""


class SatadjNonConvergence(MoistStepFailure):
    """Saturation adjustment ran out of iterations (CM1 stops the run)."""


class CourantStop(MoistStepFailure):
    """The advective Courant number reached 1.5 or is not finite."""


class StepPhase(str, Enum):
    CLOSURE = "closure"
    HELD_TENDENCIES = "solve1-held-tendencies"
    PRE_ACOUSTIC = "pre-acoustic"
    ACOUSTIC = "acoustic"
    POST_ACOUSTIC = "post-acoustic"
    SCALAR_MOIST = "scalar-moist-rk"
    REMOVE_HELD_EOS = "remove-held-and-moist-eos"
    MASS_BEGIN = "dry-mass-reduction"
    MOMENTUM_BOUNDARIES = "momentum-boundaries"
    SCALAR_BOUNDARIES = "scalar-boundaries"
    TKE = "tke-rk"
    MASS_FINISH = "dry-mass-correction"
    PDEFQ = "positive-definite-moisture"
    MICROPHYSICS = "microphysics"
    POST_PHYSICS = "post-physics-eos"
    SOLVE3 = "solve3"


@dataclass(frozen=True, slots=True)
class ScheduledOperation:
    phase: StepPhase
    nrk: int | None


@functools.lru_cache(maxsize=1)
def large_step_schedule() -> tuple[ScheduledOperation, ...]:
    """CM1 r21.1 solve1 -> solve2 -> mp_driver -> solve3 chronology."""
    order = [ScheduledOperation(StepPhase.CLOSURE, None), ScheduledOperation(StepPhase.HELD_TENDENCIES, None)]
    for nrk in (1, 2, 3):
        order.extend(ScheduledOperation(p, nrk) for p in (StepPhase.PRE_ACOUSTIC, StepPhase.ACOUSTIC,
                                                          StepPhase.POST_ACOUSTIC, StepPhase.SCALAR_MOIST))
        if nrk == 3:
            order.extend((ScheduledOperation(StepPhase.REMOVE_HELD_EOS, nrk),
                          ScheduledOperation(StepPhase.MASS_BEGIN, nrk)))
        order.append(ScheduledOperation(StepPhase.MOMENTUM_BOUNDARIES, nrk))
        if nrk < 3:
            order.append(ScheduledOperation(StepPhase.SCALAR_BOUNDARIES, nrk))
        order.append(ScheduledOperation(StepPhase.TKE, nrk))
        if nrk == 3:
            order.append(ScheduledOperation(StepPhase.MASS_FINISH, nrk))
    order.extend(ScheduledOperation(p, None) for p in (StepPhase.PDEFQ, StepPhase.MICROPHYSICS,
                                                       StepPhase.POST_PHYSICS, StepPhase.SOLVE3))
    return tuple(order)


# operations that may follow SCALAR_MOIST in the same stage's concurrent tail
# (REMOVE_HELD_EOS / MASS_BEGIN / MASS_FINISH take no separate work here)
TAIL_PHASES = frozenset({StepPhase.MOMENTUM_BOUNDARIES, StepPhase.SCALAR_BOUNDARIES, StepPhase.TKE,
                         StepPhase.REMOVE_HELD_EOS, StepPhase.MASS_BEGIN, StepPhase.MASS_FINISH})


@dataclass(frozen=True, slots=True)
class StretchedColumnSpec:
    """CM1 stretch_z = 1 parameters of a vertically stretched column
    (param.F:7814-8139 as build_vertical_levels restates it): the physical
    top, the heights where the stretching starts and ends, and the layer
    depths below and above; MoistStepConfig.dz is the coordinate's
    reference dz (rdz = 1/dz)."""

    ztop_m: float
    str_bot_m: float
    str_top_m: float
    dz_bot_m: float
    dz_top_m: float


# The 640x768x80 supercell column: 20 m at the ground to 500 m aloft, lid
# at 20.8 km, reference dz 100 m.
SUPERCELL_STRETCHED_COLUMN = StretchedColumnSpec(20800.0, 200.0, 15800.0, 20.0, 500.0)


@dataclass(frozen=True, slots=True)
class MoistStepConfig:
    ni: int
    nj: int
    nk: int
    dx: float
    dy: float
    dz: float
    dt: float
    nsound: int
    alph: float = 0.60
    kdiv: float = 0.10
    lateral_sides: tuple[int, int, int, int] = (2, 2, 2, 2)
    # None: the uniform column (the terrain operator family on flat metrics);
    # a spec: the flat (terrain_flag=.false.) family on that stretched column
    column: StretchedColumnSpec | None = None
    # the final-RK dry-air mass correction (CM1 apmasscon = 1, the supercell
    # namelist's): between the pre-physics equation of state and the Kessler
    # driver, against the state's mass1 ledger
    apmasscon: bool = True
    # the SGS stress and scalar diffusion held tendencies (CM1 gettau and
    # turbu/turbv/turbw added into the momentum tendencies of every RK
    # stage; turbs of theta and the moisture rows into the held theta and
    # moisture tendencies): the flat texts on a stretched column, the
    # terrain texts on the uniform one
    sgs_diffusion: bool = False
    # CM1's upper Rayleigh damping, irdamp = 1 (held u, v, w and theta
    # tendencies toward the base state above rayleigh_zd_m at rate
    # rayleigh_rdalpha; the supercell namelist's zd and rdalpha)
    rayleigh: bool = False
    # CM1's dissipative heating (idiss = 1, the supercell namelist's): the
    # TKE closure's dissipation rate heats theta through the held tendency
    dissipative_heating: bool = False
    rayleigh_zd_m: float = 15000.0
    rayleigh_rdalpha: float = 3.3333333333e-3

    @property
    def obc(self) -> int:
        w, e, s, n = self.lateral_sides
        return w | (e << 4) | (s << 8) | (n << 12)

    @property
    def stretched(self) -> bool:
        return self.column is not None

    def vertical_levels(self):
        """The CM1 vertical coordinate of the column (stretch_z 1 when a
        column spec is set, else the uniform coordinate)."""
        from .vertical import build_vertical_levels, uniform_vertical_levels

        if self.column is None:
            return uniform_vertical_levels(self.nk, self.dz)
        c = self.column
        return build_vertical_levels(stretch_z=1, nk=self.nk, dz_m=self.dz, ztop_m=c.ztop_m, str_bot_m=c.str_bot_m,
                                     str_top_m=c.str_top_m, dz_bot_m=c.dz_bot_m, dz_top_m=c.dz_top_m)


NUMQ = 3  # Kessler: qv, qc, qr
# per-species scratch of the moisture advection and pdef chain
SPECIES_SCRATCH = ("moisture_padded", "fx", "fy", "fz", "advx", "advy", "advz", "candidate")
# theta + the moisture species, momentum/pressure boundaries, TKE
SIDE_STREAMS = 1 + NUMQ + 2
QROWS = 6  # the eqtset2 terms and calcnm read six mass rows (the last three zero)


def moist_state_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    """Every array of the composed state (float32 unless named in
    MOIST_STATE_DTYPES)."""
    ng = 3
    su, sv = (nk + 2, nj + 2 * ng, ni + 1 + 2 * ng), (nk + 2, nj + 1 + 2 * ng, ni + 2 * ng)
    sw, ss, pr = (nk + 3, nj + 2 * ng, ni + 2 * ng), (nk + 2, nj + 2 * ng, ni + 2 * ng), (nk + 2, nj + 2, ni + 2)
    mass, face, plane = (nk, nj, ni), (nk + 1, nj, ni), (nj, ni)
    s: dict[str, tuple[int, ...]] = {}
    for n in ("ua", "u3d", "uten", "rru"):
        s[n] = su
    for n in ("va", "v3d", "vten", "rrv"):
        s[n] = sv
    for n in ("wa", "w3d", "wten", "rrw", "fz"):
        s[n] = sw
    s["fx"], s["fy"] = su, sv
    for n in ("ppi", "pp3d", "ppx", "ppd", "piadv", "ppterm", "ppten", "thv", "qk", "pk1", "pk2", "mm", "fpk", "divh",
              "hadvp", "dum3", "elim_c", "elim_d"):
        s[n] = pr
    for n in COLUMN_DIAGNOSTIC_NAMES:
        s[n] = (1,)
    s.update(radbcw=(nk + 2, nj + 2 * ng), radbce=(nk + 2, nj + 2 * ng), radbcs=(nk + 2, ni + 2 * ng),
             radbcn=(nk + 2, ni + 2 * ng), uh=(ni + 2 * ng,), vh=(nj + 2 * ng,), ruf=(ni + 1 + 2 * ng,),
             rvf=(nj + 1 + 2 * ng,), scalar=ss, dum8=ss, theta_padded=ss, moisture_padded=ss)
    for n in ("th3d", "tha", "thterm", "divergence", "theta_div", "divx", "pp3d_c", "prs", "rho", "rr", "kessler_rr",
              "thheld", "qpten", "qtten", "qvten", "qcten", "theta_adv", "advx", "advy", "advz", "candidate",
              "temperature", "qt", "thv_c", "qvci", "pi0_3d", "th0_3d", "fall_velocity", "ones_mass"):
        s[n] = mass
    s["q3d"], s["qa"] = (QROWS, *mass), (QROWS, *mass)
    s["qheld"], s["moist_adv"] = (NUMQ, *mass), (NUMQ, *mass)
    s["saturation_mask"] = mass
    for n in ("rf", "nm", "defv", "defh", "tke3d", "tkea", "tketen", "tk", "grdscl", "rgrdscl", "lenscl", "dissten",
              "cme", "ce1", "ce2", "csm", "kmh", "kmv", "khh", "khv", "tke_workspace"):
        s[n] = face
    s.update(uc=(nk, nj, ni + 1), vc=(nk, nj + 1, ni), wc=face, th0=(nk,), pi0=(nk,), qv0=(nk,), rain=(1, nj, ni),
             prate=plane, asq=(3,), qbudget=(10,), ruh=(ni,), rvh=(nj,), mass1=(1,))
    return s


MOIST_STATE_DTYPES = {"saturation_mask": np.uint8, "asq": np.float64, "qbudget": np.float64, "mass1": np.float64}

METRIC_NAMES = ("terrain_msl", "zh", "zf", "mh", "rmh", "mf", "rmf", "c1", "c2", "rho0_3d", "rr0", "rf0", "rrf0", "gz",
                "rgz", "gzu", "rgzu", "gzv", "rgzv", "dzdx", "dzdy", "gx", "gxu", "gy", "gyv")


def _libm_powf():
    import ctypes
    import ctypes.util

    lib = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
    fn = lib.powf
    fn.restype, fn.argtypes = ctypes.c_float, [ctypes.c_float, ctypes.c_float]
    return fn


def startup_thermodynamics(pi0_3d, pp3d, th0_3d, th3d, qv, c1, c2):
    """prs, rho, rr and rf of a start from its pi, theta and qv, in the
    reference's startup order (cpu_startup_thermodynamics,
    src/cm1core/cuda_cartesian_startup.py:295-345; CM1 init3d): prs =
    p00*powf(pi0 + pp3d, cp/rd) with the host C library's powf, rho =
    prs/((theta*pi)*(rd + max(qv, 0)*rv)), rr = 1/rho, rf from c1/c2 inside
    and the second-order extrapolation at the two boundary faces; binary32
    one operation at a time."""
    f = np.float32
    rd, rv, p00 = f(287.04), f(461.5), f(100000.0)
    cpdrd = f(f(1005.7) / rd)
    pi = (np.asarray(pi0_3d, f) + np.asarray(pp3d, f)).astype(f)
    powf = _libm_powf()
    levels, inverse = np.unique(pi, return_inverse=True)
    pw = np.array([powf(float(x), float(cpdrd)) for x in levels], f)[inverse].reshape(pi.shape)
    prs = (p00 * pw).astype(f)
    theta = (np.asarray(th0_3d, f) + np.asarray(th3d, f)).astype(f)
    gas = (rd + (np.maximum(f(0.0), np.asarray(qv, f)) * rv).astype(f)).astype(f)
    rho = (prs / ((theta * pi).astype(f) * gas).astype(f)).astype(f)
    rr = (f(1.0) / rho).astype(f)
    nk = rho.shape[0]
    rf = np.zeros((nk + 1,) + rho.shape[1:], f)
    rf[1:nk] = ((c1[1:nk] * rho[:-1]).astype(f) + (c2[1:nk] * rho[1:]).astype(f)).astype(f)
    rf[0] = _extrap(rho[0], rho[1], rho[2])
    rf[nk] = _extrap(rho[nk - 1], rho[nk - 2], rho[nk - 3])
    return prs, rho, rr, rf


def _extrap(a, b, c):
    f = np.float32
    s = ((f(1.875) * a).astype(f) + (f(-1.25) * b).astype(f)).astype(f)
    return (s + (f(0.375) * c).astype(f)).astype(f)


def weisman_klemp_initial_state(cfg: MoistStepConfig, *, seed: int = 0, bubble_k: float = 3.0,
                                noise_k: float = 0.1, bubble_radius_m: tuple[float, float] = (10000.0, 1400.0),
                                bubble_center_z_m: float = 1400.0, bubble_cloud: float = 0.0,
                                bubble_rain: float = 0.0,
                                bubble_offset_m: tuple[float, float] = (0.0, 0.0)) -> tuple[dict[str, np.ndarray],
                                                                            dict[str, np.ndarray]]:
    """Host (numpy float32) state and flat terrain metrics of a
    Weisman-Klemp supercell start on cfg's grid: the isnd = 5 column
    (theta, qv, pi on the mass heights), the quarter-circle hodograph, a
    cos^2 warm bubble at the domain centre (shifted by bubble_offset_m in x
    and y) plus seeded uniform noise of
    +-noise_k, cloud and rain water bubble_cloud / bubble_rain (kg/kg) in
    the bubble's core (r < 1/2), TKE at its floor, zero radiation
    histories."""
    from .analytic_state import analytic_shear_u, analytic_shear_v, weisman_klemp_column

    ni, nj, nk = cfg.ni, cfg.nj, cfg.nk
    f = np.float32
    shapes = moist_state_shapes(ni, nj, nk)
    s = {n: np.zeros(sh, dtype=MOIST_STATE_DTYPES.get(n, np.float32)) for n, sh in shapes.items()}
    levels = cfg.vertical_levels() if cfg.stretched else None
    zh = np.asarray(levels.zh[1:nk + 1], f) if levels is not None else \
        ((np.arange(nk, dtype=np.float64) + 0.5) * cfg.dz).astype(f)
    col = weisman_klemp_column(zh, 1)
    s["th0"][:], s["pi0"][:], s["qv0"][:] = col.theta_k, col.pi, col.qv_kg_per_kg
    s["th0_3d"][:] = s["th0"][:, None, None]
    s["pi0_3d"][:] = s["pi0"][:, None, None]
    s["prs"][:] = col.pressure_pa[:, None, None]
    u0 = analytic_shear_u(zh).astype(f)
    v0 = analytic_shear_v(zh).astype(f)
    s["u3d"][1:nk + 1] = u0[:, None, None]
    s["v3d"][1:nk + 1] = v0[:, None, None]
    rng = np.random.default_rng(seed)
    x = (np.arange(ni) + 0.5) * cfg.dx - 0.5 * ni * cfg.dx - bubble_offset_m[0]
    y = (np.arange(nj) + 0.5) * cfg.dy - 0.5 * nj * cfg.dy - bubble_offset_m[1]
    r = np.sqrt((x[None, None, :] / bubble_radius_m[0]) ** 2 + (y[None, :, None] / bubble_radius_m[0]) ** 2 +
                ((zh.astype(np.float64)[:, None, None] - bubble_center_z_m) / bubble_radius_m[1]) ** 2)
    bubble = np.where(r < 1.0, bubble_k * np.cos(0.5 * np.pi * r) ** 2, 0.0)
    s["th3d"][:] = (bubble + rng.uniform(-noise_k, noise_k, (nk, nj, ni))).astype(f)
    s["q3d"][0] = s["qv0"][:, None, None]
    s["q3d"][1] = np.where(r < 0.5, bubble_cloud, 0.0).astype(f)
    s["q3d"][2] = np.where(r < 0.5, bubble_rain, 0.0).astype(f)
    s["tke3d"][1:nk] = f(1.0e-4)
    for n in ("uh", "vh", "ruf", "rvf", "ruh", "rvh", "ones_mass"):
        s[n][:] = f(1.0)
    # the density of the start from its pi, theta and qv (the reference's
    # startup thermodynamics); the metrics' c1/c2 then give rf
    zero = np.zeros((nk + 1, nj, ni), f)
    _, rho0, _, _ = startup_thermodynamics(s["pi0_3d"], s["pp3d_c"], s["th0_3d"], s["th3d"], s["q3d"][0], zero, zero)
    m = flat_metrics(cfg, rho0) if levels is None else stretched_metrics(cfg, levels, rho0)
    prs, rho, rr, rf = startup_thermodynamics(s["pi0_3d"], s["pp3d_c"], s["th0_3d"], s["th3d"], s["q3d"][0], m["c1"],
                                              m["c2"])
    s["prs"][:], s["rho"][:], s["rr"][:], s["rf"][:] = prs, rho, rr, rf
    # the base-state winds and the upper damping profiles (CM1 irdamp = 1
    # above the configuration's zd, param.F:8631-8673)
    from .rayleigh import build_rayleigh_coefficients

    m["u0"], m["v0"] = u0.copy(), v0.copy()
    m["tauh"], m["taus"], m["tauf"] = build_rayleigh_coefficients(m["zh"][:, 0, 0], m["zf"][:, 0, 0],
                                                                  damping_start_m=cfg.rayleigh_zd_m)
    for cur, base in (("ua", "u3d"), ("va", "v3d"), ("wa", "w3d"), ("tha", "th3d"), ("qa", "q3d"), ("tkea", "tke3d"),
                      ("ppi", "pp3d")):
        s[cur][:] = s[base]
    return s, m


def flat_metrics(cfg: MoistStepConfig, rho: np.ndarray) -> dict[str, np.ndarray]:
    """Terrain metrics of a flat uniform column: gz = 1, zero slopes, c1 =
    c2 = 1/2, base density from the initial moist density's column means."""
    from .terrain_open import terrain_static_shapes

    ni, nj, nk = cfg.ni, cfg.nj, cfg.nk
    f = np.float32
    sh = terrain_static_shapes(ni=ni, nj=nj, nk=nk)
    m = {n: np.zeros(s, f) for n, s in sh.items()}
    for n in ("mh", "rmh", "mf", "rmf", "gz", "rgz", "gzu", "rgzu", "gzv", "rgzv"):
        m[n][:] = f(1.0)
    m["c1"][:], m["c2"][:] = f(0.5), f(0.5)
    m["zh"][:] = ((np.arange(nk) + 0.5) * cfg.dz).astype(f)[:, None, None]
    m["zf"][:] = (np.arange(nk + 1) * cfg.dz).astype(f)[:, None, None]
    prof = rho.astype(np.float64).mean(axis=(1, 2)).astype(f)
    m["rho0_3d"][:] = prof[:, None, None]
    m["rr0"][:] = (f(1.0) / m["rho0_3d"]).astype(f)
    rf = np.empty(nk + 1, f)
    rf[1:nk] = (f(0.5) * prof[:-1] + f(0.5) * prof[1:]).astype(f)
    rf[0], rf[nk] = prof[0], prof[nk - 1]
    m["rf0"][:] = rf[:, None, None]
    m["rrf0"][:] = (f(1.0) / m["rf0"]).astype(f)
    return m


def column_c1_c2(zh: np.ndarray, zf: np.ndarray, nk: int) -> tuple[np.ndarray, np.ndarray]:
    """Face interpolation weights of a column from its CM1-indexed mass
    heights zh (nk+2, ghosts at 0 and nk+1) and face heights zf (nk+3):
    c2(k) = (zf(k) - zh(k-1)) / (zh(k) - zh(k-1)), c1 = 1 - c2, at faces
    k = 1..nk+1 (the reconstruction of rust/cm1-state/src/child_auxiliary.rs:1043-1050)."""
    f = np.float32
    c2 = np.empty(nk + 1, f)
    for k in range(1, nk + 2):
        c2[k - 1] = (f(zf[k]) - f(zh[k - 1])) / (f(zh[k]) - f(zh[k - 1]))
    return (f(1.0) - c2).astype(f), c2


def padded_base_density(rho0: np.ndarray) -> np.ndarray:
    """(nk+2, nj+6, ni+6) base density of the padded lane: the interior
    rho0_3d, each halo column and row repeating the nearest edge, each ghost
    level the nearest interior level."""
    nk, nj, ni = rho0.shape
    p = np.zeros((nk + 2, nj + 6, ni + 6), np.float32)
    p[1:nk + 1, 3:nj + 3, 3:ni + 3] = rho0
    p[1:nk + 1, 3:nj + 3, :3] = rho0[:, :, :1]
    p[1:nk + 1, 3:nj + 3, ni + 3:] = rho0[:, :, -1:]
    p[:, :3, :] = p[:, 3:4, :]
    p[:, nj + 3:, :] = p[:, nj + 2:nj + 3, :]
    p[0], p[nk + 1] = p[1], p[nk]
    return p


def stretched_metrics(cfg: MoistStepConfig, levels, rho: np.ndarray) -> dict[str, np.ndarray]:
    """Metrics of a flat stretched column: gz = 1, zero slopes, the
    generated coordinate's mh/mf/rmh/rmf broadcast over the plane, c1/c2 from
    its heights, base density from the initial moist density's level means;
    plus the column profiles the flat operators read (mh_profile nk+2 words,
    mf_profile nk+3, CM1-indexed) and the padded base density rho0_padded."""
    from .terrain_open import terrain_static_shapes

    ni, nj, nk = cfg.ni, cfg.nj, cfg.nk
    f = np.float32
    m = {n: np.zeros(sh, f) for n, sh in terrain_static_shapes(ni=ni, nj=nj, nk=nk).items()}
    for n in ("gz", "rgz", "gzu", "rgzu", "gzv", "rgzv"):
        m[n][:] = f(1.0)
    mh, mf = np.asarray(levels.mh, f), np.asarray(levels.mf, f)
    rmh, rmf = np.asarray(levels.rmh, f), np.asarray(levels.rmf, f)
    m["mh"][:], m["rmh"][:] = mh[1:nk + 1, None, None], rmh[1:nk + 1, None, None]
    m["mf"][:], m["rmf"][:] = mf[1:nk + 2, None, None], rmf[1:nk + 2, None, None]
    zh, zf = np.asarray(levels.zh, f), np.asarray(levels.zf, f)
    c1, c2 = column_c1_c2(zh, zf, nk)
    m["c1"][:], m["c2"][:] = c1[:, None, None], c2[:, None, None]
    m["zh"][:] = zh[1:nk + 1, None, None]
    m["zf"][:] = zf[1:nk + 2, None, None]
    prof = rho.astype(np.float64).mean(axis=(1, 2)).astype(f)
    m["rho0_3d"][:] = prof[:, None, None]
    m["rr0"][:] = (f(1.0) / m["rho0_3d"]).astype(f)
    rf = np.empty(nk + 1, f)
    rf[1:nk] = (c1[1:nk] * prof[:-1] + c2[1:nk] * prof[1:]).astype(f)
    rf[0], rf[nk] = prof[0], prof[nk - 1]
    m["rf0"][:] = rf[:, None, None]
    m["rrf0"][:] = (f(1.0) / m["rf0"]).astype(f)
    m["mh_profile"], m["mf_profile"] = mh.copy(), mf.copy()
    m["rho0_padded"] = padded_base_density(m["rho0_3d"])
    return m


class MoistLargeStep:
    """The composed moist large step on one CUDA device.  ``state`` and
    ``metrics`` are dicts of device tensors with moist_state_shapes /
    terrain_static_shapes; everything is enqueued on ``stream`` (the current
    stream when None) and nothing synchronises, so a whole step can be
    captured in a CUDA graph."""

    def __init__(self, cfg: MoistStepConfig, state: dict[str, torch.Tensor], metrics: dict[str, torch.Tensor], *,
                 stream: Any | None = None, concurrent: bool = True, tuner: Any | None = None) -> None:
        self.cfg, self.s, self.m = cfg, state, metrics
        self.stream = stream
        # the scalar advection's z-chunk per stage kind (fifth order, WENO5);
        # None: the kernel's default, else picked for this grid by ``tuner``
        # (gm1_b200.autotune.Autotuner) at the end of set-up
        self.chunk = {False: None, True: None}
        ni, nj, nk = cfg.ni, cfg.nj, cfg.nk
        s, m = state, metrics
        self.k3 = dict(ni=ni, nj=nj, nk=nk)
        self.grid = dict(ni=ni, nj=nj, nk=nk, dx=cfg.dx, dy=cfg.dy, dz=cfg.dz)
        # views the operators take as whole arrays
        self.q_rows = [s["q3d"][r] for r in range(NUMQ)]
        self.qa_rows = [s["qa"][r] for r in range(NUMQ)]
        self.tke_arrays = {"tkea": s["tkea"], "tke3d": s["tke3d"], "tketen": s["tketen"], "kmh": s["kmh"],
                           "kmv": s["kmv"], "rho": s["rho"], "rf": s["rf"], "mh": m["mh"], "mf": m["mf"],
                           "gz": m["gz"], "rgz": m["rgz"], "rgzu": m["rgzu"], "rgzv": m["rgzv"], "c1": m["c1"],
                           "c2": m["c2"], "rrf0": m["rrf0"], "rru": s["rru"], "rrv": s["rrv"], "rrw": s["rrw"],
                           "divx": s["divx"]}
        self.sgs_arrays = {"ruh": s["ruh"], "rvh": s["rvh"], "rmf": m["rmf"], **{n: s[n] for n in (
            "nm", "defv", "defh", "tkea", "tk", "grdscl", "rgrdscl", "lenscl", "dissten", "cme", "ce1", "ce2", "csm",
            "kmh", "kmv", "khh", "khv", "tketen")}}
        self.def_arrays = {"u3d": s["uc"], "v3d": s["vc"], "w3d": s["wc"], "rho": s["rho"], "rf": s["rf"],
                           **{n: m[n] for n in ("c1", "c2", "gz", "rgz", "gzu", "rgzu", "gzv", "rgzv", "gx", "gy")},
                           "defv": s["defv"], "defh": s["defh"]}
        self.nm_arrays = {"c1": m["c1"], "c2": m["c2"], "mf": m["mf"], "pi0": s["pi0"], "th0": s["th0"],
                          "prs": s["prs"], "pp3d": s["pp3d_c"], "th3d": s["th3d"], "q3d": s["q3d"], "nm": s["nm"],
                          "temperature": s["temperature"], "qt": s["qt"], "thv": s["thv_c"], "qvci": s["qvci"],
                          "saturation_mask": s["saturation_mask"]}
        self.held_arrays = {"th0": s["th0_3d"], "pi0": s["pi0_3d"], "rho": s["rho"], "ppi": s["pp3d_c"],
                            "tha": s["tha"], "qa": s["qa"], "qpten": s["qpten"], "qtten": s["qtten"],
                            "qvten": s["qvten"], "qcten": s["qcten"], "thheld": s["thheld"], "qheld": s["qheld"],
                            "ppten": s["ppten"]}
        self.post_arrays = {"rru": s["rru"], "rrv": s["rrv"], "rrw": s["rrw"], "rgzu": m["rgzu"], "rgzv": m["rgzv"],
                            "dzdx": m["dzdx"], "dzdy": m["dzdy"], "gz": m["gz"], "rho0_3d": m["rho0_3d"],
                            "rf0": m["rf0"], "thterm": s["thterm"], "divergence": s["divergence"],
                            "theta_divergence_term": s["theta_div"], "divx": s["divx"]}
        # Each moisture species has its own packing and pdef scratch (species 0
        # uses the state's), so the species can advect concurrently; fresh
        # scratch starts at zero as the state's does.
        self.species_scratch = [{n: s[n] for n in SPECIES_SCRATCH}] + [
            {n: torch.zeros_like(s[n]) for n in SPECIES_SCRATCH} for _ in range(1, NUMQ)]
        self.chain_arrays = [{"scalar_a": self.qa_rows[r], "scalar_padded": self.species_scratch[r]["moisture_padded"],
                              "rho0_3d": m["rho0_3d"], "gz": m["gz"], "rgz": m["rgz"], "rr0": m["rr0"], "c1": m["c1"],
                              "c2": m["c2"], "divx": s["divx"], "rru": s["rru"], "rrv": s["rrv"], "rrw": s["rrw"],
                              **{n: self.species_scratch[r][n] for n in SPECIES_SCRATCH if n != "moisture_padded"},
                              "advection": s["moist_adv"][r]}
                             for r in range(NUMQ)]
        # side streams of the concurrent step (created here so that a CUDA
        # graph capture of step() can fork onto them)
        dev = s["u3d"].device
        self.concurrent = concurrent
        self._side = [torch.cuda.Stream(dev) for _ in range(SIDE_STREAMS)] if concurrent else []
        if cfg.apmasscon:
            # init3d.F:2483-2527: the initial dry-air mass of the state, unless
            # it carries one (a restored ledger)
            with torch.cuda.stream(torch.cuda.current_stream(s["rho"].device) if stream is None else stream):
                dry_mass(s["rho"], s["ruh"], s["rvh"], m["rmh"], ni=ni, nj=nj, nk=nk, out=s["mass1"],
                         only_if_unset=True)
        self.kessler = create_cuda_gm1_kessler_large_step_transition(
            {"ruh": s["ruh"], "rvh": s["rvh"], "rmh": m["rmh"], "mh": m["mh"], "pi0": s["pi0_3d"], "th0": s["th0_3d"],
             "rr": s["kessler_rr"], "rho": s["rho"], "pp3d": s["pp3d_c"], "th3d": s["th3d"], "prs": s["prs"],
             "qv": self.q_rows[0], "qc": self.q_rows[1], "qr": self.q_rows[2], "fall_velocity": s["fall_velocity"],
             "rain": s["rain"], "prate": s["prate"], "asq": s["asq"], "qbudget": s["qbudget"]},
            **self.grid, dt=cfg.dt, selection=Gm1KesslerDriverSelection(equation_set=2), stream=stream,
            carriers=Gm1KesslerHeldCarriers(s["qpten"], s["qtten"], s["qvten"], s["qcten"]),
            mass1=s["mass1"] if cfg.apmasscon else None)
        from .momentum import _Arrays as _MomArrays, _Column, _lib as _mom_lib, _STRUCT as _MOM

        self._mom_lib = _mom_lib()
        self._mom = _MomArrays(**{n: (s[n] if n in s else m[n]).data_ptr() for n in _MOM})
        self._tos_lib = _tos_lib()
        self._tos = _TosArrays(**{n: s[n].data_ptr() for n in TOS_ARRAY_NAMES})
        self._tos_m = _TosMetrics(**{n: m[n].data_ptr() for n in TOS_METRICS})
        self.flat = cfg.stretched
        if self.flat:
            # the flat (terrain_flag=.false.) family on the stretched column:
            # the column profiles, the reference rdz, the padded base density
            from .advection import StretchedColumn
            from .momentum import StretchedMomentumColumn

            self.rdz = float(np.float32(np.float32(1.0) / np.float32(cfg.dz)))
            for n, shape in (("mh_profile", (nk + 2,)), ("mf_profile", (nk + 3,)),
                             ("rho0_padded", (nk + 2, nj + 6, ni + 6))):
                if n not in m or tuple(m[n].shape) != shape:
                    raise ValueError(f"a stretched-column step needs metrics[{n!r}] of shape {shape}")
            self._column = _Column(1, m["rho0_padded"].data_ptr(), None, None, None, None, 0.0,
                                   m["mh_profile"].data_ptr(), m["mf_profile"].data_ptr(), m["rr0"].data_ptr(),
                                   self.rdz)
            self.scalar_column = StretchedColumn(True, mh=m["mh_profile"], rdz=self.rdz)
            self.post_column = StretchedMomentumColumn(True, m["rho0_padded"], mh=m["mh_profile"], rdz=self.rdz)
            self.flat_def_arrays = {"u3d": s["uc"], "v3d": s["vc"], "w3d": s["wc"], "rho": s["rho"], "rf": s["rf"],
                                    "mf": m["mf"], "c1": m["c1"], "c2": m["c2"], "defv": s["defv"],
                                    "defh": s["defh"]}
            self.flat_turbt_arrays = {"tke3d": s["tke3d"], "kmh": s["kmh"], "kmv": s["kmv"], "rho": s["rho"],
                                      "rf": s["rf"], "mh": m["mh"], "mf": m["mf"], "tketen": s["tketen"]}
            self.flat_stage_arrays = {"tkea": s["tkea"], "tke3d": s["tke3d"], "tketen": s["tketen"], "c2": m["c2"],
                                      "rrf0": m["rrf0"], "rru": s["rru"], "rrv": s["rrv"], "rrw": s["rrw"],
                                      "divx": s["divx"]}
        if cfg.sgs_diffusion:
            # the flat texts on a stretched column, the terrain texts on the
            # uniform one (its flat metrics: gz = 1, zero slopes)
            from .stress import (STRAIN_NAMES, TAU_NAMES, TERRAIN_METRIC_NAMES, flat_stress_shapes,
                                 scalar_turbulence_workspace, terrain_scalar_turbulence_workspace)

            shp = flat_stress_shapes(ni, nj, nk)
            self.stress = {n: torch.zeros(shp[n], dtype=torch.float32, device=dev)
                           for n in STRAIN_NAMES + TAU_NAMES + ("uten", "vten", "wten")}
            self.stress_arrays = {"u3d": s["uc"], "v3d": s["vc"], "w3d": s["wc"], "rho": s["rho"], "rf": s["rf"],
                                  "mh": m["mh"], "mf": m["mf"], "kmh": s["kmh"], "kmv": s["kmv"], **self.stress}
            self.turbs_arrays = {"th0": s["th0"], "tha": s["tha"], "qa": s["qa"], "rho": s["rho"], "rr": s["rr"],
                                 "rf": s["rf"], "mh": m["mh"], "mf": m["mf"], "khh": s["khh"], "khv": s["khv"],
                                 "thten1": s["thheld"], "qten": s["qheld"]}
            if self.flat:
                self.stress_arrays["mh_profile"] = m["mh_profile"]
                self.turbs_arrays["workspace"] = scalar_turbulence_workspace(ni, nj, nk, NUMQ, dev)
            else:
                metrics = {n: m[n] for n in TERRAIN_METRIC_NAMES}
                self.stress_arrays.update(metrics)
                self.turbs_arrays.update(metrics)
                self.turbs_arrays["workspace"] = terrain_scalar_turbulence_workspace(ni, nj, nk, NUMQ, dev)
        if cfg.rayleigh and not cfg.sgs_diffusion:
            from .stress import flat_stress_shapes as _shapes

            shp = _shapes(ni, nj, nk)
            self.stress = {n: torch.zeros(shp[n], dtype=torch.float32, device=dev) for n in ("uten", "vten", "wten")}
        if cfg.rayleigh:
            for n in ("u0", "v0", "tauh", "taus", "tauf"):
                if n not in m:
                    raise ValueError(f"a damped step needs metrics[{n!r}] (the builder's base-state winds and tau)")
            self.rayleigh_arrays = {"tauh": m["tauh"], "taus": m["taus"], "tauf": m["tauf"], "u0": m["u0"],
                                    "v0": m["v0"], "ua": s["uc"], "va": s["vc"], "wa": s["wc"][:nk], "tha": s["tha"],
                                    "uten1": self.stress["uten"], "vten1": self.stress["vten"],
                                    "wten1": self.stress["wten"][:nk], "thten1": s["thheld"]}
        # failure words folded on the device every step (gm1b_step_status_fold)
        self.status_acc = torch.zeros(8, dtype=torch.int32, device=dev)
        self._courant = torch.zeros(1, dtype=torch.float32, device=dev)
        self._courant_keys = torch.zeros(nk, dtype=torch.int32, device=dev)
        self._ones_i = torch.ones(ni, dtype=torch.float32, device=dev)
        self._ones_j = torch.ones(nj, dtype=torch.float32, device=dev)
        self._mh_col = m["mh"][:, 0, 0].contiguous()
        self.completed_steps = 0
        if tuner is not None:
            self._tune(tuner)

    def _tune(self, tuner) -> None:
        """The z-chunk of the fifth-order and the WENO5 scalar advection for
        this grid shape: each candidate timed on the state's theta carrier
        into a scratch tendency (the state is not written); the chunk changes
        which CTA forms which level, not a word."""
        s, m, cfg = self.s, self.m, self.cfg
        st = self._st()
        scratch = torch.empty_like(s["theta_adv"])
        flux = {"rru": s["rru"], "rrv": s["rrv"], "rrw": s["rrw"]}
        met = {"c1": m["c1"], "c2": m["c2"], "rr0": m["rr0"], "gz": m["gz"]}
        kind = "moist_scalar_advection5" + ("_flat" if self.flat else "")
        with torch.cuda.stream(st):
            for weno in (False, True):
                def run(c, weno=weno):
                    self.chunk[weno] = c
                    self._advect(s["theta_padded"], flux, met, scratch, theta_weps_f64(), 3 if weno else 1, st)
                self.chunk[weno] = tuner.choose(kind + ("_weno" if weno else ""), cfg.ni, cfg.nj, cfg.nk, run)

    # -- helpers -----------------------------------------------------------
    def _st(self):
        dev = self.s["u3d"].device
        return torch.cuda.current_stream(dev) if self.stream is None else self.stream

    def _interior_pp3d_to_compact(self) -> None:
        nk, nj, ni = self.cfg.nk, self.cfg.nj, self.cfg.ni
        self.s["pp3d_c"].copy_(self.s["pp3d"][1:nk + 1, 1:nj + 1, 1:ni + 1])

    def _compact_pp3d_to_interior(self) -> None:
        nk, nj, ni = self.cfg.nk, self.cfg.nj, self.cfg.ni
        self.s["pp3d"][1:nk + 1, 1:nj + 1, 1:ni + 1].copy_(self.s["pp3d_c"])

    # -- phases ------------------------------------------------------------
    def closure(self) -> None:
        s, cfg, st = self.s, self.cfg, self._st()
        nk, nj, ni = cfg.nk, cfg.nj, cfg.ni
        with torch.cuda.stream(st):
            s["uc"].copy_(s["u3d"][1:nk + 1, 3:3 + nj, 3:4 + ni])
            s["vc"].copy_(s["v3d"][1:nk + 1, 3:4 + nj, 3:3 + ni])
            s["wc"].copy_(s["w3d"][1:nk + 2, 3:3 + nj, 3:3 + ni])
            self._interior_pp3d_to_compact()
        self._fold_courant(st)
        launch_cuda_moist_nm(self.nm_arrays, **self.k3, dz=cfg.dz, stream=st)
        if self.flat:
            launch_cuda_flat_deformation(self.flat_def_arrays, mh_profile=self.m["mh_profile"], **self.k3, dx=cfg.dx,
                                         dy=cfg.dy, rdz=self.rdz, stream=st)
        else:
            launch_cuda_terrain_deformation(self.def_arrays, **self.grid, stream=st)
        launch_cuda_sgs_tke(self.sgs_arrays, **self.grid, stream=st)
        with torch.cuda.stream(st):
            s["tke3d"].copy_(s["tkea"])
        if self.flat:
            launch_cuda_flat_tke_diffusion(self.flat_turbt_arrays, **self.k3, dx=cfg.dx, dy=cfg.dy, rdz=self.rdz,
                                           dt=cfg.dt, stream=st)
        else:
            launch_cuda_tke_diffusion(self.tke_arrays, **self.grid, dt=cfg.dt, stream=st)
        if cfg.sgs_diffusion:
            self._held_stress(st)
        elif cfg.rayleigh:
            with torch.cuda.stream(st):
                for n in ("uten", "vten", "wten"):
                    self.stress[n].zero_()

    def _held_stress(self, st) -> None:
        """The held momentum tendencies: zeroed, then the SGS stress added
        (the closure's held phase, cuda_cartesian_closure.py:1202-1291, with
        neither damper on so the Rayleigh terms are zero)."""
        from .stress import launch_cuda_flat_sgs_stress, launch_cuda_terrain_sgs_stress

        cfg = self.cfg
        with torch.cuda.stream(st):
            for n in ("uten", "vten", "wten"):
                self.stress[n].zero_()
        if self.flat:
            launch_cuda_flat_sgs_stress(self.stress_arrays, **self.k3, dx=cfg.dx, dy=cfg.dy, rdz=self.rdz, dt=cfg.dt,
                                        stream=st)
        else:
            launch_cuda_terrain_sgs_stress(self.stress_arrays, **self.k3, dx=cfg.dx, dy=cfg.dy, dz=cfg.dz,
                                           dt=cfg.dt, stream=st)

    def held_tendencies(self) -> None:
        s, st = self.s, self._st()
        with torch.cuda.stream(st):
            s["thheld"].zero_()
            s["qheld"].zero_()
        if self.cfg.rayleigh:
            # the damping added into the held momentum (uten1 + uten of the
            # closure's held sum) and assigned to the held theta before the
            # scalar diffusion adds to it (solve1.F:412-454)
            from .rayleigh import launch_cuda_rayleigh_held

            launch_cuda_rayleigh_held(self.rayleigh_arrays, **self.k3, rdalpha=self.cfg.rayleigh_rdalpha,
                                      profiles=True, add_momentum=True, stream=st)
        if self.cfg.dissipative_heating:
            # idiss: after the damping and before the subgrid turbulence
            # (solve1.F:917-975)
            from .stress import launch_cuda_dissipative_heating

            launch_cuda_dissipative_heating({"dissten": s["dissten"], "pi0": s["pi0"], "ppi": s["pp3d_c"],
                                             "qa": s["qa"], "thten1": s["thheld"]}, **self.k3, stream=st)
        if self.cfg.sgs_diffusion:
            # turbs for theta and the moisture rows into the held thten1/qten
            # the eqtset 2 composition then reads (solve1.F:1169-1233)
            from .stress import launch_cuda_flat_scalar_turbulence, launch_cuda_terrain_scalar_turbulence

            cfg = self.cfg
            turbs = launch_cuda_flat_scalar_turbulence if self.flat else launch_cuda_terrain_scalar_turbulence
            turbs(self.turbs_arrays, **self.k3, numq=NUMQ, dx=cfg.dx, dy=cfg.dy, dz=cfg.dz, dt=cfg.dt, stream=st)
        mo.held_compose(self.held_arrays, **self.k3, dt=self.cfg.dt, stream=st)

    def pre_acoustic(self, nrk: int) -> None:
        s, m, cfg, st = self.s, self.m, self.cfg, self._st()
        launch_cuda_eqtset2_stage_terms(**self.k3, th0=s["th0"], qv0=s["qv0"], pi0=s["pi0"], th3d=s["th3d"],
                                        q3d=s["q3d"], pp3d=s["pp3d"], thv=s["thv"], ppterm=s["ppterm"],
                                        buoyancy=s["dum8"], thterm=s["thterm"], piadv=s["piadv"], stream=st)
        mo.open_fill(s["thv"], "pressure", **self.k3, stream=st)
        mo.open_fill(s["dum8"], "scalar", **self.k3, stream=st)
        with torch.cuda.stream(st):
            s["uten"].zero_()
            s["vten"].zero_()
            s["wten"].zero_()
            if cfg.sgs_diffusion or cfg.rayleigh:
                # the held momentum seeds the stage tendencies' physical cells
                # (pack_cartesian_held_momentum, cuda_cartesian_dynamics.py:206)
                nk, nj, ni = cfg.nk, cfg.nj, cfg.ni
                s["uten"][1:nk + 1, 3:3 + nj, 3:4 + ni].copy_(self.stress["uten"])
                s["vten"][1:nk + 1, 3:4 + nj, 3:3 + ni].copy_(self.stress["vten"])
                s["wten"][1:nk + 2, 3:3 + nj, 3:3 + ni].copy_(self.stress["wten"])
        if self.flat:
            # solve2.F:484-487 (bcwsfc, bc2d of w(1)) and :575 (bcw(rrw,0)) are
            # terrain_flag statements: a flat column runs neither
            _native.check(self._mom_lib.gm1b_momentum_advection5_column(
                cfg.ni, cfg.nj, cfg.nk, ctypes.byref(self._mom), cfg.obc, cfg.dx, cfg.dy, ctypes.byref(self._column),
                ctypes.c_void_p(st.cuda_stream)), "gm1b_momentum_advection5_column")
            mo.moist_buoyancy_flat(s["dum8"], m["c1"], m["c2"], s["wten"], **self.k3, stream=st)
            return
        if nrk >= 2:
            mo.bcwsfc(s["u3d"], s["v3d"], s["w3d"], m["gz"], m["dzdx"], m["dzdy"], **self.k3, stream=st)
            mo.w_level1_fill(s["w3d"], **self.k3, stream=st)
        args = (cfg.ni, cfg.nj, cfg.nk, ctypes.byref(self._mom), cfg.obc, cfg.dx, cfg.dy, cfg.dz,
                ctypes.c_void_p(st.cuda_stream))
        _native.check(self._mom_lib.gm1b_momentum_mass_flux5(*args), "gm1b_momentum_mass_flux5")
        mo.open_fill(s["rrw"], "w_keep_ends", **self.k3, stream=st)
        _native.check(self._mom_lib.gm1b_momentum_transport5(*args), "gm1b_momentum_transport5")
        mo.moist_buoyancy(s["dum8"], m["c1"], m["c2"], m["gxu"], m["gyv"], s["uten"], s["vten"], s["wten"],
                          **self.k3, stream=st)

    def acoustic(self, nrk: int) -> None:
        cfg, st = self.cfg, self._st()
        stage_without_fills = 255 & ~128
        if self.flat:
            _native.check(self._tos_lib.gm1b_terrain_open_stage_column(
                cfg.ni, cfg.nj, cfg.nk, nrk, cfg.dt, cfg.nsound, cfg.dx, cfg.dy, float(np.float32(cfg.alph)),
                float(np.float32(cfg.kdiv)), stage_without_fills, 0, cfg.obc, ctypes.byref(self._tos),
                ctypes.byref(self._tos_m), ctypes.byref(self._column), ctypes.c_void_p(st.cuda_stream)),
                "gm1b_terrain_open_stage_column")
            return
        _native.check(self._tos_lib.gm1b_terrain_open_stage(
            cfg.ni, cfg.nj, cfg.nk, nrk, cfg.dt, cfg.nsound, cfg.dx, cfg.dy, cfg.dz, float(np.float32(cfg.alph)),
            float(np.float32(cfg.kdiv)), stage_without_fills, 0, ctypes.byref(self._tos), ctypes.byref(self._tos_m),
            ctypes.c_void_p(st.cuda_stream)), "gm1b_terrain_open_stage")

    def post_acoustic(self, nrk: int) -> None:
        if self.flat:
            cfg = self.cfg
            mo.post_acoustic_flux_column(self.post_arrays, self.post_column, **self.k3, dx=cfg.dx, dy=cfg.dy,
                                         stream=self._st())
            return
        mo.post_acoustic_flux(self.post_arrays, **self.grid, stream=self._st())

    def _theta_advection(self, nrk: int, st) -> None:
        s, m, cfg = self.s, self.m, self.cfg
        flux = {"rru": s["rru"], "rrv": s["rrv"], "rrw": s["rrw"]}
        met = {"c1": m["c1"], "c2": m["c2"], "rr0": m["rr0"], "gz": m["gz"]}
        theta_transport_scalar(s["th0"], s["th3d"], s["theta_padded"], **self.k3, stream=st)
        mo.open_fill(s["theta_padded"], "scalar", **self.k3, stream=st)
        with torch.cuda.stream(st):
            s["theta_adv"].zero_()
        self._advect(s["theta_padded"], flux, met, s["theta_adv"], theta_weps_f64(), nrk, st)

    def _advect(self, padded, flux, met, tendency, weps, nrk: int, st) -> None:
        s, cfg = self.s, self.cfg
        if self.flat:
            launch_cuda_gm1_child_stretched_scalar_advection5(padded, flux, met, s["divx"], tendency, None,
                                                              self.scalar_column, **self.k3, dx=cfg.dx, dy=cfg.dy,
                                                              nrk=nrk, weps=weps, stream=st,
                                                              lateral_sides=cfg.lateral_sides, write_fluxes=False,
                                                              levels_per_chunk=self.chunk[nrk == 3])
        else:
            launch_cuda_scalar_advection5(padded, flux, met, s["divx"], tendency, None, weps=weps, **self.grid,
                                          nrk=nrk, stream=st, lateral_sides=cfg.lateral_sides, write_fluxes=False,
                                          levels_per_chunk=self.chunk[nrk == 3])

    def _species_advection(self, r: int, nrk: int, st) -> None:
        s, m, cfg = self.s, self.m, self.cfg
        padded = self.species_scratch[r]["moisture_padded"]
        mo.pack_scalar(self.q_rows[r], padded, **self.k3, stream=st)
        mo.open_fill(padded, "scalar", **self.k3, stream=st)
        with torch.cuda.stream(st):
            s["moist_adv"][r].zero_()
        weps = moisture_weps_f64(r)
        if nrk < 3:
            self._advect(padded, {"rru": s["rru"], "rrv": s["rrv"], "rrw": s["rrw"]},
                         {"c1": m["c1"], "c2": m["c2"], "rr0": m["rr0"], "gz": m["gz"]}, s["moist_adv"][r], weps, nrk,
                         st)
        elif self.flat:
            mo.pdef_moisture_chain_column(self.chain_arrays[r], self.scalar_column, **self.k3, dx=cfg.dx, dy=cfg.dy,
                                          dttmp=scalar_moist_rk_stage_timestep_f32(cfg.dt, nrk), weps=weps,
                                          lateral_obc=cfg.obc, pdefweno=0 if r == 0 else 1, stream=st)
        else:
            mo.pdef_moisture_chain(self.chain_arrays[r], **self.grid,
                                   dttmp=scalar_moist_rk_stage_timestep_f32(cfg.dt, nrk), weps=weps,
                                   lateral_obc=cfg.obc, pdefweno=0 if r == 0 else 1, stream=st)

    def scalar_moist(self, nrk: int) -> None:
        """theta and the moisture species advect (concurrently, each on its own
        side stream, when the step is concurrent), then one RK compose."""
        s, cfg, st = self.s, self.cfg, self._st()
        if self.concurrent:
            lanes = self._side[:1 + NUMQ]
            self._fork(st, lanes)
            self._theta_advection(nrk, lanes[0])
            for r in range(NUMQ):
                self._species_advection(r, nrk, lanes[1 + r])
            self._join(st, lanes)
        else:
            self._theta_advection(nrk, st)
            for r in range(NUMQ):
                self._species_advection(r, nrk, st)
        compose_scalar_moist_rk_stage(s["tha"], s["qa"][:NUMQ], s["thheld"], s["qheld"], s["theta_div"],
                                      s["theta_adv"], s["moist_adv"], s["th3d"], s["q3d"][:NUMQ], nrk=nrk, dt=cfg.dt,
                                      stream=st)

    def momentum_boundaries(self, nrk: int) -> None:
        s, m, st = self.s, self.m, self._st()
        mo.open_fill(s["u3d"], "u", **self.k3, stream=st)
        mo.open_fill(s["v3d"], "v", **self.k3, stream=st)
        mo.open_fill(s["w3d"], "w", **self.k3, stream=st)
        if not self.flat:  # solve2.F:1676: bcwsfc is a terrain_flag statement
            mo.bcwsfc(s["u3d"], s["v3d"], s["w3d"], m["gz"], m["dzdx"], m["dzdy"], **self.k3, stream=st)

    def scalar_boundaries(self, nrk: int) -> None:
        mo.open_fill(self.s["pp3d"], "pressure", **self.k3, stream=self._st())

    def tke_rk(self, nrk: int) -> None:
        if self.flat:
            cfg = self.cfg
            launch_cuda_flat_tke_rk_stage(self.flat_stage_arrays, mf_profile=self.m["mf_profile"],
                                          workspace=self.s["tke_workspace"], **self.k3, nrk=nrk, dx=cfg.dx,
                                          dy=cfg.dy, rdz=self.rdz, dt=cfg.dt, stream=self._st())
            return
        launch_cuda_tke_rk_stage(self.tke_arrays, workspace=self.s["tke_workspace"], **self.grid, nrk=nrk,
                                 dt=self.cfg.dt, stream=self._st())

    def microphysics(self) -> None:
        st = self._st()
        with torch.cuda.stream(st):
            self._interior_pp3d_to_compact()
        self.kessler.stream = st
        self.kessler.apply()
        self.fold_kessler_status(st)
        with torch.cuda.stream(st):
            self._compact_pp3d_to_interior()

    def solve3(self) -> None:
        s, m, st = self.s, self.m, self._st()
        with torch.cuda.stream(st):
            s["ppx"].add_(s["pp3d"])
            for cur, base in (("ua", "u3d"), ("va", "v3d"), ("wa", "w3d"), ("ppi", "pp3d"), ("tha", "th3d"),
                              ("qa", "q3d"), ("tkea", "tke3d")):
                s[cur].copy_(s[base])
        mo.solve3_density(s["rho"], m["c1"], m["c2"], s["rr"], s["rf"], **self.k3, stream=st)

    # -- failure words -----------------------------------------------------
    def _fold_courant(self, st) -> None:
        """The advective Courant number of the compact winds uc/vc/wc (the
        state entering this step), folded into status_acc."""
        cfg, s = self.cfg, self.s
        advective_courant_number(u=s["uc"], v=s["vc"], w=s["wc"], uh=self._ones_i, vh=self._ones_j,
                                 mh=self._mh_col, dt_s=cfg.dt, dx_m=cfg.dx, dy_m=cfg.dy, dz_m=cfg.dz,
                                 level_keys=self._courant_keys, stream=st, out=self._courant)
        _native.check(_native.lib().gm1b_step_status_fold(
            None, ctypes.c_void_p(self._courant.data_ptr()), ctypes.c_void_p(self.status_acc.data_ptr()),
            ctypes.c_void_p(st.cuda_stream)), "gm1b_step_status_fold")

    def fold_kessler_status(self, stream: Any | None = None) -> None:
        """Fold the Kessler operator's status words (those of its last run
        in the step's workspace) into status_acc; microphysics() calls it
        after the transition."""
        st = self._st() if stream is None else stream
        _native.check(_native.lib().gm1b_step_status_fold(
            ctypes.c_void_p(self.kessler.workspace.status.data_ptr()), None,
            ctypes.c_void_p(self.status_acc.data_ptr()), ctypes.c_void_p(st.cuda_stream)), "gm1b_step_status_fold")

    def status(self) -> dict[str, Any]:
        """Waits for the enqueued work and reads the folded failure words of
        every step since construction (or the last reset_status())."""
        st = self._st()
        st.synchronize()
        acc = self.status_acc.cpu().numpy()
        return {"satadj_nonconverged_cells": int(acc[0]), "max_fall_substeps": int(acc[1]),
                "blown_up_fall_columns": int(acc[2]),
                "max_courant": float(acc[3:4].view(np.float32)[0]) if acc[4] else None,
                "courant_samples": int(acc[4]), "kessler_samples": int(acc[5])}

    def reset_status(self) -> None:
        with torch.cuda.stream(self._st()):
            self.status_acc.zero_()

    def check(self, *, current_state: bool = True) -> dict[str, Any]:
        """Refuse the integration as the reference does: raise
        SatadjNonConvergence if any saturation adjustment ran out of
        iterations (or a fall column blew up) and CourantStop if the
        advective Courant number reached 1.5 or is not finite
        (src/cm1core/cuda_cartesian_finish.py:638-639;
        src/cm1core/gm1_runtime.py:518-549).  The Courant number covers the
        state entering every step taken and, with current_state, the
        current state too."""
        if current_state:
            cfg, s, st = self.cfg, self.s, self._st()
            nk, nj, ni = cfg.nk, cfg.nj, cfg.ni
            with torch.cuda.stream(st):
                s["uc"].copy_(s["u3d"][1:nk + 1, 3:3 + nj, 3:4 + ni])
                s["vc"].copy_(s["v3d"][1:nk + 1, 3:4 + nj, 3:3 + ni])
                s["wc"].copy_(s["w3d"][1:nk + 2, 3:3 + nj, 3:3 + ni])
            self._fold_courant(st)
        out = self.status()
        if out["satadj_nonconverged_cells"] or out["blown_up_fall_columns"]:
            raise SatadjNonConvergence(
                f"GM1 Kessler satadj failed to converge in 100 iterations in {out['satadj_nonconverged_cells']} "
                f"cells ({out['blown_up_fall_columns']} rain columns with a non-finite fall Courant number)")
        c = out["max_courant"]
        if c is not None and (not np.isfinite(c) or c >= CM1_COURANT_STOP):
            raise CourantStop(f"the advective Courant number {c!r} has reached CM1's stop value "
                              f"{CM1_COURANT_STOP} or is not finite (misclibs.F:2714)")
        return out

    # -- driver ------------------------------------------------------------
    def execute(self, op: ScheduledOperation) -> None:
        p, nrk = op.phase, op.nrk
        if p is StepPhase.CLOSURE:
            self.closure()
        elif p is StepPhase.HELD_TENDENCIES:
            self.held_tendencies()
        elif p is StepPhase.PRE_ACOUSTIC:
            self.pre_acoustic(nrk)
        elif p is StepPhase.ACOUSTIC:
            self.acoustic(nrk)
        elif p is StepPhase.POST_ACOUSTIC:
            self.post_acoustic(nrk)
        elif p is StepPhase.SCALAR_MOIST:
            self.scalar_moist(nrk)
        elif p is StepPhase.MOMENTUM_BOUNDARIES:
            self.momentum_boundaries(nrk)
        elif p is StepPhase.SCALAR_BOUNDARIES:
            self.scalar_boundaries(nrk)
        elif p is StepPhase.TKE:
            self.tke_rk(nrk)
        elif p is StepPhase.MICROPHYSICS:
            self.microphysics()
        elif p is StepPhase.SOLVE3:
            self.solve3()
        # REMOVE_HELD_EOS and POST_PHYSICS are the first and last parts of
        # the Kessler transition (MICROPHYSICS); nothing between them reads
        # or writes its fields.  MASS_BEGIN / MASS_FINISH (dry-mass
        # correction) and PDEFQ (the Kessler operator's own pdefq runs inside
        # it) take no separate work here.

    # -- concurrency -------------------------------------------------------
    @staticmethod
    def _fork(main, lanes) -> None:
        ev = torch.cuda.Event()
        ev.record(main)
        for ln in lanes:
            ln.wait_event(ev)

    @staticmethod
    def _join(main, lanes) -> None:
        for ln in lanes:
            ev = torch.cuda.Event()
            ev.record(ln)
            main.wait_event(ev)

    def _stage_tail(self, ops) -> None:
        """SCALAR_MOIST, MOMENTUM_BOUNDARIES, SCALAR_BOUNDARIES and TKE of one
        RK stage touch disjoint fields (scalars and moisture / u, v, w and
        pi' / TKE; all read the same mass fluxes), so they run concurrently:
        the scalars on the main stream (forking its own side streams), the
        boundaries and TKE on two more, joined before the next stage."""
        main = self._st()
        bnd, tke = self._side[1 + NUMQ], self._side[2 + NUMQ]
        self._fork(main, (bnd, tke))
        saved = self.stream
        for op in ops:
            if op.phase in (StepPhase.MOMENTUM_BOUNDARIES, StepPhase.SCALAR_BOUNDARIES):
                self.stream = bnd
            elif op.phase is StepPhase.TKE:
                self.stream = tke
            else:
                self.stream = main
            try:
                self.execute(op)
            finally:
                self.stream = saved
        self._join(main, (bnd, tke))

    def _run_ops(self, ops) -> None:
        """Operations of the schedule in order (each stage's scalar /
        boundary / TKE tail concurrently when the step is concurrent)."""
        q = 0
        while q < len(ops):
            op = ops[q]
            if self.concurrent and op.phase is StepPhase.SCALAR_MOIST:
                tail = [op]
                q += 1
                while q < len(ops) and ops[q].nrk == op.nrk and ops[q].phase in TAIL_PHASES:
                    tail.append(ops[q])
                    q += 1
                self._stage_tail(tail)
                continue
            self.execute(op)
            q += 1

    def step(self) -> None:
        """One large step: the operations of large_step_schedule() in order."""
        self._run_ops(large_step_schedule())
        self.completed_steps += 1

    # -- a step split at the dry-mass ledger (a domain decomposed over
    # subdomains forms the ledger over all of them between the halves) -----
    def _microphysics_index(self) -> int:
        ops = large_step_schedule()
        return next(q for q, op in enumerate(ops) if op.phase is StepPhase.MICROPHYSICS)

    def step_begin(self, window: tuple[int, int, int, int], partials: torch.Tensor) -> None:
        """The step up to the dry-mass ledger: every operation before the
        microphysics, then the Kessler transition's held removal and
        pre-physics EOS and the level partials of the cells in window
        (i0, i1, j0, j1) into partials."""
        if not self.cfg.apmasscon:
            raise RuntimeError("step_begin/step_end split the dry-mass correction: the configuration has none")
        self._run_ops(large_step_schedule()[:self._microphysics_index()])
        st = self._st()
        with torch.cuda.stream(st):
            self._interior_pp3d_to_compact()
        self.kessler.stream = st
        self.kessler.begin(window, partials)

    def step_end(self, partials: torch.Tensor, cells: int) -> None:
        """The rest of the step from the added partials of the domain's
        `cells` cells: the correction, the Kessler driver and recapture, the
        operations after the microphysics."""
        st = self._st()
        self.kessler.stream = st
        self.kessler.end(partials, cells)
        self.fold_kessler_status(st)
        with torch.cuda.stream(st):
            self._compact_pp3d_to_interior()
        self._run_ops(large_step_schedule()[self._microphysics_index() + 1:])
        self.completed_steps += 1


def upload(host: dict[str, np.ndarray], device: torch.device | str = "cuda") -> dict[str, torch.Tensor]:
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(device) for k, v in host.items()}


# ---------------------------------------------------------------------------
# the same step through the C ABI's whole-step entry point
# ---------------------------------------------------------------------------
# gm1b_moist_state, in the header's order (the species scratch of species 1
# and 2 last)
NATIVE_STATE_NAMES = (
    "ua", "u3d", "uten", "rru", "va", "v3d", "vten", "rrv", "wa", "w3d", "wten", "rrw", "fz", "fx", "fy",
    "ppi", "pp3d", "ppx", "ppd", "piadv", "ppterm", "ppten", "thv", "qk", "pk1", "pk2", "mm", "fpk", "divh", "hadvp",
    "dum3", "elim_c", "elim_d",
    "tri_aa", "tri_bb", "tri_cc", "tri_dd", "tri_pivot", "tri_residual",
    "radbcw", "radbce", "radbcs", "radbcn", "uh", "vh", "ruf", "rvf", "scalar", "dum8", "theta_padded",
    "moisture_padded",
    "th3d", "tha", "thterm", "divergence", "theta_div", "divx", "pp3d_c", "prs", "rho", "rr", "kessler_rr", "thheld",
    "qpten", "qtten", "qvten", "qcten", "theta_adv", "advx", "advy", "advz", "candidate", "temperature", "qt",
    "thv_c", "qvci", "pi0_3d", "th0_3d", "fall_velocity", "ones_mass",
    "q3d", "qa", "qheld", "moist_adv",
    "rf", "nm", "defv", "defh", "tke3d", "tkea", "tketen", "tk", "grdscl", "rgrdscl", "lenscl", "dissten", "cme",
    "ce1", "ce2", "csm", "kmh", "kmv", "khh", "khv", "tke_workspace",
    "uc", "vc", "wc", "th0", "pi0", "qv0", "rain", "prate", "ruh", "rvh",
    "saturation_mask", "asq", "qbudget",
) + tuple(f"{n}_{r}" for r in (1, 2) for n in ("moisture_padded", "fx", "fy", "fz", "advx", "advy", "advz",
                                                 "candidate")) + ("mass1",)
NATIVE_METRIC_NAMES = METRIC_NAMES + ("mh_profile", "mf_profile", "rho0_padded", "u0", "v0", "tauh", "taus",
                                      "tauf")


class _NativeState(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in NATIVE_STATE_NAMES]


class _NativeMetrics(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in NATIVE_METRIC_NAMES]


class _NativeConfig(ctypes.Structure):
    _fields_ = [("ni", ctypes.c_int32), ("nj", ctypes.c_int32), ("nk", ctypes.c_int32), ("dx", ctypes.c_float),
                ("dy", ctypes.c_float), ("dz", ctypes.c_float), ("dt", ctypes.c_float), ("nsound", ctypes.c_int32),
                ("alph", ctypes.c_float), ("kdiv", ctypes.c_float), ("lateral_sides", ctypes.c_int32 * 4),
                ("stretched", ctypes.c_int32), ("concurrent", ctypes.c_int32), ("apmasscon", ctypes.c_int32),
                ("sgs_diffusion", ctypes.c_int32), ("rayleigh", ctypes.c_int32), ("rdalpha", ctypes.c_float),
                ("dissipative_heating", ctypes.c_int32)]


def _native_lib():
    lib = _native.lib()
    if not getattr(lib, "_mls_bound", False):
        c = ctypes
        lib.gm1b_moist_step_create.argtypes = [c.POINTER(_NativeConfig), c.POINTER(_NativeState),
                                               c.POINTER(_NativeMetrics), c.POINTER(c.c_void_p)]
        lib.gm1b_moist_step_create.restype = c.c_int32
        lib.gm1b_moist_large_step.argtypes = [c.c_void_p, c.c_void_p]
        lib.gm1b_moist_large_step.restype = c.c_int32
        lib.gm1b_moist_step_status.argtypes = [c.c_void_p, c.POINTER(c.c_int32), c.c_int32, c.c_void_p]
        lib.gm1b_moist_step_status.restype = c.c_int32
        lib.gm1b_moist_step_destroy.argtypes = [c.c_void_p]
        lib.gm1b_moist_step_destroy.restype = c.c_int32
        lib._mls_bound = True
    return lib


class NativeMoistLargeStep:
    """The composed moist large step through the C ABI's whole-step entry
    point (gm1b_moist_step_create / gm1b_moist_large_step): one library call
    per step, the same launches in the same order as MoistLargeStep, so the
    two leave the same words.  ``state`` and ``metrics`` are the device dicts
    MoistLargeStep takes; the scratch of moisture species 1 and 2 is
    allocated here (zero), everything else is the caller's."""

    def __init__(self, cfg: MoistStepConfig, state: dict[str, torch.Tensor], metrics: dict[str, torch.Tensor], *,
                 stream: Any | None = None, concurrent: bool = True) -> None:
        self.cfg, self.s, self.m, self.stream = cfg, state, metrics, stream
        self.scratch = {f"{n}_{r}": torch.zeros_like(state[n]) for r in (1, 2) for n in SPECIES_SCRATCH}
        arrays = {**state, **self.scratch}
        missing = [n for n in NATIVE_STATE_NAMES if n not in arrays]
        if missing:
            raise ValueError(f"missing moist-step arrays: {', '.join(missing)}")
        for n in NATIVE_STATE_NAMES:
            t = arrays[n]
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()):
                raise ValueError(f"{n} must be a contiguous CUDA tensor")
        self._state = _NativeState(**{n: arrays[n].data_ptr() for n in NATIVE_STATE_NAMES})
        self._metrics = _NativeMetrics(**{n: (metrics[n].data_ptr() if n in metrics else None)
                                          for n in NATIVE_METRIC_NAMES})
        self._config = _NativeConfig(cfg.ni, cfg.nj, cfg.nk, cfg.dx, cfg.dy, cfg.dz, cfg.dt, cfg.nsound,
                                     float(np.float32(cfg.alph)), float(np.float32(cfg.kdiv)),
                                     (ctypes.c_int32 * 4)(*cfg.lateral_sides), 1 if cfg.stretched else 0,
                                     1 if concurrent else 0, 1 if cfg.apmasscon else 0,
                                     1 if cfg.sgs_diffusion else 0, 1 if cfg.rayleigh else 0,
                                     float(np.float32(cfg.rayleigh_rdalpha)),
                                     1 if cfg.dissipative_heating else 0)
        lib = _native_lib()
        handle = ctypes.c_void_p()
        with torch.cuda.device(state["u3d"].device):
            _native.check(lib.gm1b_moist_step_create(ctypes.byref(self._config), ctypes.byref(self._state),
                                                     ctypes.byref(self._metrics), ctypes.byref(handle)),
                          "gm1b_moist_step_create")
        self._handle = handle
        self.completed_steps = 0

    def _st(self):
        dev = self.s["u3d"].device
        return torch.cuda.current_stream(dev) if self.stream is None else self.stream

    def step(self) -> None:
        _native.check(_native_lib().gm1b_moist_large_step(self._handle, ctypes.c_void_p(self._st().cuda_stream)),
                      "gm1b_moist_large_step")
        self.completed_steps += 1

    def status(self, *, reset: bool = False) -> tuple[int, dict[str, Any]]:
        out = (ctypes.c_int32 * 8)()
        rc = _native_lib().gm1b_moist_step_status(self._handle, out, 1 if reset else 0,
                                                  ctypes.c_void_p(self._st().cuda_stream))
        if rc < 0:
            _native.check(rc, "gm1b_moist_step_status")
        words = np.array(out[:], np.int32)
        return rc, {"satadj_nonconverged_cells": int(words[0]), "max_fall_substeps": int(words[1]),
                    "blown_up_fall_columns": int(words[2]),
                    "max_courant": float(words[3:4].view(np.float32)[0]) if words[4] else None,
                    "courant_samples": int(words[4]), "kessler_samples": int(words[5])}

    def check(self) -> dict[str, Any]:
        """Refuse as the reference does (SatadjNonConvergence, CourantStop)
        on the failure words folded over every step taken."""
        rc, out = self.status()
        if rc == 1:
            raise SatadjNonConvergence(f"GM1 Kessler satadj failed to converge ({out})")
        if rc == 2:
            raise CourantStop(f"the advective Courant number {out['max_courant']!r} reached CM1's stop value")
        return out

    def close(self) -> None:
        if getattr(self, "_handle", None):
            _native_lib().gm1b_moist_step_destroy(self._handle)
            self._handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
