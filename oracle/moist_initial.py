"""Weisman-Klemp moist starting states for the oracle composition - TEST
INFRASTRUCTURE ONLY.

The CPU baseline and the reference arm of the benchmark build their inputs
here, from the oracle's own restatement of the initial column
(init_oracle.c: weisman_klemp_column_with_iterations and analytic_shear_u/v,
rust/cm1-state/src/storm_initialization.rs:194,354,373) and NumPy, so that
nothing on those paths loads the CUDA library.  The state is the one the
package's weisman_klemp_initial_state builds for the same arguments, word for
word (tests/test_oracle_moist_step.py checks it): the isnd = 5 column on the
mass heights, the quarter-circle hodograph, a cos^2 warm bubble plus seeded
uniform noise from numpy.random.default_rng(seed), optional cloud and rain
in the bubble's core, TKE at its floor, flat terrain metrics whose base
density is the initial moist density's level means.
"""

from __future__ import annotations

import numpy as np

from oracle.initial import analytic_shear, wk_column

NUMQ = 3
QROWS = 6
NG = 3
DIAGNOSTIC_NAMES = ("tri_aa", "tri_bb", "tri_cc", "tri_dd", "tri_pivot", "tri_residual")
DTYPES = {"saturation_mask": np.uint8, "asq": np.float64, "qbudget": np.float64, "mass1": np.float64}


def terrain_static_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    """Terrain/metric arrays of the padded lane (terrain_static_shapes of the
    reference's src/cm1core/cuda_terrain_open_boundary.py)."""
    mass, face, plane = (nk, nj, ni), (nk + 1, nj, ni), (nj, ni)
    return {"terrain_msl": plane, "zh": mass, "zf": face, "mh": mass, "rmh": mass, "mf": face, "rmf": face,
            "c1": face, "c2": face, "rho0_3d": mass, "rr0": mass, "rf0": face, "rrf0": face, "gz": plane,
            "rgz": plane, "gzu": (nj, ni + 1), "rgzu": (nj, ni + 1), "gzv": (nj + 1, ni), "rgzv": (nj + 1, ni),
            "dzdx": plane, "dzdy": plane, "gx": face, "gxu": (nk + 1, nj, ni + 1), "gy": face,
            "gyv": (nk + 1, nj + 1, ni)}


def moist_state_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    """Every array of the composed moist state (the package's
    moist_state_shapes)."""
    su, sv = (nk + 2, nj + 2 * NG, ni + 1 + 2 * NG), (nk + 2, nj + 1 + 2 * NG, ni + 2 * NG)
    sw, ss, pr = (nk + 3, nj + 2 * NG, ni + 2 * NG), (nk + 2, nj + 2 * NG, ni + 2 * NG), (nk + 2, nj + 2, ni + 2)
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
    for n in DIAGNOSTIC_NAMES:
        s[n] = (1,)
    s.update(radbcw=(nk + 2, nj + 2 * NG), radbce=(nk + 2, nj + 2 * NG), radbcs=(nk + 2, ni + 2 * NG),
             radbcn=(nk + 2, ni + 2 * NG), uh=(ni + 2 * NG,), vh=(nj + 2 * NG,), ruf=(ni + 1 + 2 * NG,),
             rvf=(nj + 1 + 2 * NG,), scalar=ss, dum8=ss, theta_padded=ss, moisture_padded=ss)
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


def flat_metrics(ni: int, nj: int, nk: int, dz: float, rho: np.ndarray) -> dict[str, np.ndarray]:
    """Flat uniform-column metrics: gz = 1, zero slopes, c1 = c2 = 1/2, base
    density from the initial moist density's level means."""
    f = np.float32
    m = {n: np.zeros(s, f) for n, s in terrain_static_shapes(ni, nj, nk).items()}
    for n in ("mh", "rmh", "mf", "rmf", "gz", "rgz", "gzu", "rgzu", "gzv", "rgzv"):
        m[n][:] = f(1.0)
    m["c1"][:], m["c2"][:] = f(0.5), f(0.5)
    m["zh"][:] = ((np.arange(nk) + 0.5) * dz).astype(f)[:, None, None]
    m["zf"][:] = (np.arange(nk + 1) * dz).astype(f)[:, None, None]
    prof = rho.astype(np.float64).mean(axis=(1, 2)).astype(f)
    m["rho0_3d"][:] = prof[:, None, None]
    m["rr0"][:] = (f(1.0) / m["rho0_3d"]).astype(f)
    rf = np.empty(nk + 1, f)
    rf[1:nk] = (f(0.5) * prof[:-1] + f(0.5) * prof[1:]).astype(f)
    rf[0], rf[nk] = prof[0], prof[nk - 1]
    m["rf0"][:] = rf[:, None, None]
    m["rrf0"][:] = (f(1.0) / m["rf0"]).astype(f)
    return m


def column_levels(cfg) -> dict[str, np.ndarray]:
    """The oracle's stretch_z = 1 coordinate of cfg.column (reference dz =
    cfg.dz), CM1-indexed profiles."""
    from oracle.vertical import vertical_levels

    c = cfg.column
    rc, lv = vertical_levels(1, cfg.nk, cfg.dz, c.ztop_m, c.str_bot_m, c.str_top_m, c.dz_bot_m, c.dz_top_m)
    if rc != 0:
        raise ValueError(f"oracle_vertical_levels refused the column ({rc})")
    return lv


def padded_base_density(rho0: np.ndarray) -> np.ndarray:
    """(nk+2, nj+6, ni+6) base density: halo columns/rows repeat the edge,
    ghost levels the nearest interior level."""
    nk, nj, ni = rho0.shape
    p = np.zeros((nk + 2, nj + 6, ni + 6), np.float32)
    p[1:nk + 1, 3:nj + 3, 3:ni + 3] = rho0
    p[1:nk + 1, 3:nj + 3, :3] = rho0[:, :, :1]
    p[1:nk + 1, 3:nj + 3, ni + 3:] = rho0[:, :, -1:]
    p[:, :3, :] = p[:, 3:4, :]
    p[:, nj + 3:, :] = p[:, nj + 2:nj + 3, :]
    p[0], p[nk + 1] = p[1], p[nk]
    return p


def stretched_metrics(ni: int, nj: int, nk: int, lv: dict[str, np.ndarray], rho: np.ndarray) -> dict[str, np.ndarray]:
    """Metrics of a flat stretched column: the generated mh/mf/rmh/rmf over
    the plane, c2(k) = (zf(k) - zh(k-1)) / (zh(k) - zh(k-1)) and c1 = 1 - c2,
    base density from the initial density's level means, the column profiles
    and the padded base density."""
    f = np.float32
    m = {n: np.zeros(sh, f) for n, sh in terrain_static_shapes(ni, nj, nk).items()}
    for n in ("gz", "rgz", "gzu", "rgzu", "gzv", "rgzv"):
        m[n][:] = f(1.0)
    m["mh"][:], m["rmh"][:] = lv["mh"][1:nk + 1, None, None], lv["rmh"][1:nk + 1, None, None]
    m["mf"][:], m["rmf"][:] = lv["mf"][1:nk + 2, None, None], lv["rmf"][1:nk + 2, None, None]
    zh, zf = lv["zh"], lv["zf"]
    c2 = np.empty(nk + 1, f)
    for k in range(1, nk + 2):
        c2[k - 1] = (zf[k] - zh[k - 1]) / (zh[k] - zh[k - 1])
    c1 = (f(1.0) - c2).astype(f)
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
    m["mh_profile"], m["mf_profile"] = lv["mh"].copy(), lv["mf"].copy()
    m["rho0_padded"] = padded_base_density(m["rho0_3d"])
    return m


def weisman_klemp_initial_state(cfg, *, seed: int = 0, bubble_k: float = 3.0, noise_k: float = 0.1,
                                bubble_radius_m: tuple[float, float] = (10000.0, 1400.0),
                                bubble_center_z_m: float = 1400.0, bubble_cloud: float = 0.0,
                                bubble_rain: float = 0.0, bubble_offset_m: tuple[float, float] = (0.0, 0.0)):
    """(state, metrics) of a Weisman-Klemp start on cfg's grid (cfg has ni,
    nj, nk, dx, dy, dz and, for a stretched column, column)."""
    ni, nj, nk = cfg.ni, cfg.nj, cfg.nk
    f = np.float32
    s = {n: np.zeros(sh, dtype=DTYPES.get(n, np.float32)) for n, sh in moist_state_shapes(ni, nj, nk).items()}
    lv = column_levels(cfg) if getattr(cfg, "column", None) is not None else None
    zh = lv["zh"][1:nk + 1].copy() if lv is not None else ((np.arange(nk, dtype=np.float64) + 0.5) * cfg.dz).astype(f)
    col = wk_column(zh, 1)
    s["th0"][:], s["pi0"][:], s["qv0"][:] = col["th0"], col["pi0"], col["qv0"]
    s["th0_3d"][:] = s["th0"][:, None, None]
    s["pi0_3d"][:] = s["pi0"][:, None, None]
    s["prs"][:] = col["prs0"][:, None, None]
    u0, v0 = analytic_shear(zh, zh)
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
    # the density of the start from its pi, theta and qv (the reference's
    # startup thermodynamics); the metrics' c1/c2 then give rf
    s["tke3d"][1:nk] = f(1.0e-4)
    for n in ("uh", "vh", "ruf", "rvf", "ruh", "rvh", "ones_mass"):
        s[n][:] = f(1.0)
    zero = np.zeros((nk + 1, nj, ni), f)
    _, rho0, _, _ = startup_thermodynamics(s["pi0_3d"], s["pp3d_c"], s["th0_3d"], s["th3d"], s["q3d"][0], zero, zero)
    m = flat_metrics(ni, nj, nk, cfg.dz, rho0) if lv is None else stretched_metrics(ni, nj, nk, lv, rho0)
    prs, rho, rr, rf = startup_thermodynamics(s["pi0_3d"], s["pp3d_c"], s["th0_3d"], s["th3d"], s["q3d"][0], m["c1"],
                                              m["c2"])
    s["prs"][:], s["rho"][:], s["rr"][:], s["rf"][:] = prs, rho, rr, rf
    # the base-state winds and the upper damping profiles above zd
    from oracle.stress import rayleigh_coefficients

    m["u0"], m["v0"] = u0.astype(f), v0.astype(f)
    m["tauh"], m["taus"], m["tauf"] = rayleigh_coefficients(m["zh"][:, 0, 0], m["zf"][:, 0, 0],
                                                            damping_start_m=getattr(cfg, "rayleigh_zd_m", 15000.0))
    for cur, base in (("ua", "u3d"), ("va", "v3d"), ("wa", "w3d"), ("tha", "th3d"), ("qa", "q3d"), ("tkea", "tke3d"),
                      ("ppi", "pp3d")):
        s[cur][:] = s[base]
    return s, m


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
