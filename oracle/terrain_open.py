"""ctypes driver of the terrain/open acoustic-stage oracle
(terrain_open_oracle.c) - TEST INFRASTRUCTURE ONLY.  Mirrors
cpu_psolver3_terrain_open_stage_inplace and the three-stage composition
(src/cm1core/cuda_psolver3_terrain_open.py:774-913)."""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from oracle.periodic import C_REAL, REAL, load

_F = ctypes.POINTER(C_REAL)
ARRAY_NAMES = ("ppi", "pp3d", "ppx", "ppd", "piadv", "ppterm", "ppten", "thv", "qk", "pk1", "pk2", "mm", "fpk",
               "divh", "hadvp", "dum3", "elim_c", "elim_d", "tri_aa", "tri_bb", "tri_cc", "tri_dd", "tri_pivot",
               "tri_residual", "ua", "u3d", "uten", "rru", "va", "v3d", "vten", "rrv", "wa", "w3d", "wten", "rrw",
               "radbcw", "radbce", "radbcs", "radbcn", "uh", "vh", "ruf", "rvf", "scalar")
METRIC_NAMES = ("rho0_3d", "rr0", "rf0", "rrf0", "c1", "c2", "gz", "rgzu", "rgzv", "dzdx", "dzdy", "gx", "gxu", "gy",
                "gyv")
ABLATION_BITS = {"open_consumption": 1, "terrain_pressure_gradient": 2, "transformed_divergence": 4,
                 "pressure_advection": 8, "implicit_vertical_solve": 16, "between_step_pressure_fill": 32,
                 "radiation_history_production": 64, "stage_family_fills": 128}
ALL_ABLATIONS = 255


class TosArrays(ctypes.Structure):
    _fields_ = [(n, _F) for n in ARRAY_NAMES]


class TosMetrics(ctypes.Structure):
    _fields_ = [(n, _F) for n in METRIC_NAMES]


@dataclass(frozen=True)
class StageDiagnostics:
    nrk: int
    nloop: int
    dts_f32: float
    max_tridiagonal_residual: float


def _lib():
    lib = load()
    if not getattr(lib, "_tos_ready", False):
        c = ctypes
        lib.oracle_terrain_open_stage.argtypes = [c.POINTER(TosArrays), c.POINTER(TosMetrics)] + [c.c_int] * 4 + \
            [C_REAL, c.c_int, C_REAL, C_REAL, c.c_double, C_REAL, C_REAL, c.c_uint, c.POINTER(C_REAL)]
        lib.oracle_terrain_open_stage.restype = c.c_int
        lib.oracle_terrain_edge_weights.argtypes = [c.c_int, C_REAL, c.POINTER(C_REAL), c.POINTER(C_REAL)]
        lib.oracle_terrain_edge_weights.restype = None
        lib.oracle_terrain_open_stage_column.argtypes = [c.POINTER(TosArrays), c.POINTER(TosMetrics)] + \
            [c.c_int] * 4 + [C_REAL, c.c_int, C_REAL, C_REAL] + [_F] * 4 + [C_REAL, _F] + \
            [C_REAL, C_REAL, c.c_uint, c.POINTER(C_REAL)]
        lib.oracle_terrain_open_stage_column.restype = c.c_int
        lib.oracle_terrain_open_stage_flat.argtypes = [c.POINTER(TosArrays), c.POINTER(TosMetrics)] + \
            [c.c_int] * 4 + [C_REAL, c.c_int, C_REAL, C_REAL, _F, _F, C_REAL, c.c_uint] + \
            [C_REAL, C_REAL, c.c_uint, c.POINTER(C_REAL)]
        lib.oracle_terrain_open_stage_flat.restype = c.c_int
        lib._tos_ready = True
    return lib


def _bind(struct_type, names, d):
    s = struct_type()
    for n in names:
        v = d[n]
        assert v.dtype == REAL and v.flags.c_contiguous, n
        setattr(s, n, v.ctypes.data_as(_F))
    return s


def terrain_open_stage(a, m, *, ni, nj, nk, nrk, dt, nsound, dx, dy, dz, alph=0.6, kdiv=0.1,
                       ablations=ALL_ABLATIONS) -> StageDiagnostics:
    sa, sm = _bind(TosArrays, ARRAY_NAMES, a), _bind(TosMetrics, METRIC_NAMES, m)
    diag = (C_REAL * 3)()
    rc = _lib().oracle_terrain_open_stage(ctypes.byref(sa), ctypes.byref(sm), ni, nj, nk, nrk, dt, nsound, dx, dy,
                                         float(dz), alph, kdiv, ablations, diag)
    if rc != 0:
        raise ValueError(f"oracle_terrain_open_stage failed ({rc})")
    return StageDiagnostics(nrk, int(diag[0]), float(diag[1]), float(diag[2]))


def terrain_open_stage_column(a, m, column, *, ni, nj, nk, nrk, dt, nsound, dx, dy, alph=0.6, kdiv=0.1,
                              ablations=ALL_ABLATIONS) -> StageDiagnostics:
    """One stage on a stretched terrain column: ``column`` maps sigma,
    sigmaf, rds, rdsf (CM1-indexed float32 profiles), ztop and rho0p (the
    padded base density, (nk+2, nj+6, ni+6))."""
    sa, sm = _bind(TosArrays, ARRAY_NAMES, a), _bind(TosMetrics, METRIC_NAMES, m)
    prof = {n: np.ascontiguousarray(column[n], dtype=REAL) for n in ("sigma", "sigmaf", "rds", "rdsf", "rho0p")}
    assert prof["rho0p"].shape == (nk + 2, nj + 6, ni + 6)
    diag = (C_REAL * 3)()
    ptr = {n: v.ctypes.data_as(_F) for n, v in prof.items()}
    rc = _lib().oracle_terrain_open_stage_column(ctypes.byref(sa), ctypes.byref(sm), ni, nj, nk, nrk, dt, nsound, dx,
                                                dy, ptr["sigma"], ptr["sigmaf"], ptr["rds"], ptr["rdsf"],
                                                float(np.float32(column["ztop"])), ptr["rho0p"], alph, kdiv,
                                                ablations, diag)
    if rc != 0:
        raise ValueError(f"oracle_terrain_open_stage_column failed ({rc})")
    return StageDiagnostics(nrk, int(diag[0]), float(diag[1]), float(diag[2]))


def terrain_open_stage_flat(a, m, column, *, ni, nj, nk, nrk, dt, nsound, dx, dy, obc=0x2222, alph=0.6, kdiv=0.1,
                            ablations=ALL_ABLATIONS) -> StageDiagnostics:
    """One stage on a flat stretched column: ``column`` maps mh (nk+2), mf
    (nk+3) and rdz; ``obc`` packs wbc | ebc << 4 | sbc << 8 | nbc << 12."""
    sa, sm = _bind(TosArrays, ARRAY_NAMES, a), _bind(TosMetrics, METRIC_NAMES, m)
    mh = np.ascontiguousarray(column["mh"], dtype=REAL)
    mf = np.ascontiguousarray(column["mf"], dtype=REAL)
    diag = (C_REAL * 3)()
    rc = _lib().oracle_terrain_open_stage_flat(ctypes.byref(sa), ctypes.byref(sm), ni, nj, nk, nrk, dt, nsound, dx, dy,
                                              mh.ctypes.data_as(_F), mf.ctypes.data_as(_F),
                                              float(np.float32(column["rdz"])), obc, alph, kdiv, ablations, diag)
    if rc != 0:
        raise ValueError(f"oracle_terrain_open_stage_flat failed ({rc})")
    return StageDiagnostics(nrk, int(diag[0]), float(diag[1]), float(diag[2]))


def terrain_open_three_stage(a, m, **kw) -> tuple[StageDiagnostics, ...]:
    return tuple(terrain_open_stage(a, m, nrk=nrk, **kw) for nrk in (1, 2, 3))


def edge_weights(nk: int, dz: float) -> tuple[tuple[float, ...], tuple[float, ...]]:
    cgs, cgt = (C_REAL * 3)(), (C_REAL * 3)()
    _lib().oracle_terrain_edge_weights(nk, dz, cgs, cgt)
    return tuple(cgs), tuple(cgt)


def ablation_mask(**disabled: bool) -> int:
    """Mask of enabled terrain/open phases; keywords name a disabled phase
    (``open_consumption=False`` etc.), as TerrainOpenSoundAblations does."""
    mask = ALL_ABLATIONS
    for name, enabled in disabled.items():
        if not enabled:
            mask &= ~ABLATION_BITS[name]
    return mask
