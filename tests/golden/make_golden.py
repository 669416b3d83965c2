"""Generate the golden vectors of tests/golden by running the REFERENCE itself.

Run in a container where the reference source tree is present (it is read
only, never copied):

    python tests/golden/make_golden.py --reference /path/to/gm1 small
    python tests/golden/make_golden.py --reference /path/to/gm1 c1 --checkpoints 1 10

``small`` writes compressed .npz fixtures of whole input/output array sets on
small grids (operator-level raw-bit pins), ``c1`` writes SHA-256 digests of
every array of the 64x64x40 dry bubble after 1 and after N large steps of the
reference's CPU twin (a full-size pin that stays a few KB).  Inputs come from
gm1_b200.initial_state, whose digests are stored too so a test can prove it
rebuilt the same inputs.

Reference entry points used (their CPU twins, single-threaded NumPy):
  cpu_sound3_periodic_three_stage_inplace  src/cm1core/cuda_sound3_periodic.py:1071
  cpu_psolver3_trajectory_inplace          src/cm1core/cuda_psolver3_trajectory.py:761
  cpu_initial_dry_mass, cpu_apmasscon_inplace  src/cm1core/cuda_apmasscon.py:226, :256
  cpu_sgs_stress_tendency_inplace          src/cm1core/cuda_sgs_stress_tendency.py:292
  cpu_gm1_scalar_turbulence_inplace        src/cm1core/cuda_gm1_scalar_turbulence.py:414
  cpu_build_rayleigh_coefficients, cpu_rayleigh_held_inplace  src/cm1core/cuda_rayleigh_held.py:264, :213
  cpu_idiss_cell_f32                       src/cm1core/eqtset2_energy_terms.py:176
  (and the others named by each make_* function)
"""

from __future__ import annotations

import argparse
import copy
import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from gm1_b200.arrays import (  # noqa: E402
    ALL_ARRAY_NAMES,
    SOUND_ARRAY_NAMES,
    array_shapes,
    default_periodic_face_weights,
    fill_periodic_scalar_inplace,
    fill_periodic_uv_inplace,
)
from gm1_b200.initial_state import DRY_BUBBLE_64, DryBubbleCase, dry_periodic_state  # noqa: E402

ABLATION_FIELDS = (
    "momentum_advection",
    "scalar_advection",
    "base_theta_advection",
    "buoyancy",
    "post_step_ppx",
    "carrier_promotion",
)

# Small trajectory fixture: a 7x6x7 periodic box with a background wind and a
# seeded smooth perturbation so both upwind branches of every flux occur.
SMALL_CASE = DryBubbleCase(
    ni=7, nj=6, nk=7, dx=1000.0, dy=1000.0, dz=500.0, dt=0.4, nsound=6,
    bubble_radius_h=2500.0, bubble_radius_v=1500.0, bubble_center_z=1500.0,
    noise_amplitude=0.05, seed=7, u0=2.0, v0=-0.7, wind_perturbation=1.5,
)
# A second shape with nsound=8 and a larger dt, uneven ni/nj.
SMALL_CASE_B = DryBubbleCase(
    ni=9, nj=5, nk=8, dx=800.0, dy=1200.0, dz=400.0, dt=3.0, nsound=8,
    bubble_radius_h=3000.0, bubble_radius_v=1200.0, bubble_center_z=1000.0,
    noise_amplitude=0.1, seed=11, u0=-3.0, v0=1.5, wind_perturbation=2.5,
)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes(order="C")).hexdigest()


def sound_fixture(ni: int, nj: int, nk: int, seed: int) -> dict[str, np.ndarray]:
    """Horizontally varying acoustic-stage inputs satisfying the periodic
    contract of src/cm1core/cuda_sound3_periodic.py:569-602."""
    rng = np.random.default_rng(seed)
    shapes = array_shapes(ni, nj, nk)
    a = {name: np.zeros(shape, dtype=np.float32) for name, shape in shapes.items()}
    a["dtu0"], a["dtv0"] = default_periodic_face_weights(ni, nj)
    for name in ("uf", "vf", "uh", "vh"):
        a[name].fill(np.float32(1.0))
    z = (np.arange(nk + 2, dtype=np.float64) / (nk + 1))[:, None, None]
    hx = np.sin(2 * np.pi * np.arange(ni + 2) / ni)[None, None, :]
    hy = np.cos(2 * np.pi * np.arange(nj + 2) / nj)[None, :, None]
    h = 0.6 * hx + 0.3 * hy
    ones = np.ones((nk + 2, nj + 2, ni + 2))
    a["mh"][...] = (1.0 + 0.02 * z * ones).astype(np.float32)
    a["mf"][...] = (1.0 - 0.01 * z * ones).astype(np.float32)
    a["rr0"][...] = (0.9 + 0.2 * z + 0.001 * h).astype(np.float32)
    a["rf0"][...] = (1.1 - 0.15 * z + 0.001 * h).astype(np.float32)
    a["c1"][...] = (0.4 + 0.1 * z * ones).astype(np.float32)
    a["c2"][...] = (np.float32(1.0) - a["c1"]).astype(np.float32)
    a["piadv"][...] = (1.0 - 0.05 * z + 2e-5 * h).astype(np.float32)
    a["ppterm"][...] = (0.35 + 0.01 * z + 1e-4 * h).astype(np.float32)
    a["thv"][...] = (300.0 + 8.0 * z + 0.2 * h).astype(np.float32)
    a["ppten"][...] = (1e-6 * h + 5e-7 * z).astype(np.float32)
    pressure = (2e-4 * h + 4e-5 * z).astype(np.float32)
    a["ppi"][...] = pressure
    a["ppx"][...] = (0.2 * pressure + 1e-6 * z).astype(np.float32)
    for name in ("mh", "rr0", "rf0", "c1", "c2", "mf", "piadv", "ppterm", "thv", "ppten", "ppi", "ppx"):
        fill_periodic_scalar_inplace(a[name], ni=ni, nj=nj, nk=nk)
    a["ua"][1 : nk + 1, 1 : nj + 1, :] = rng.uniform(-3, 3, size=(nk, nj, ni + 1)).astype(np.float32)
    a["ua"][1 : nk + 1, 1 : nj + 1, ni] = a["ua"][1 : nk + 1, 1 : nj + 1, 0]
    a["va"][1 : nk + 1, :, 1 : ni + 1] = rng.uniform(-3, 3, size=(nk, nj + 1, ni)).astype(np.float32)
    a["va"][1 : nk + 1, nj, 1 : ni + 1] = a["va"][1 : nk + 1, 0, 1 : ni + 1]
    fill_periodic_uv_inplace(a["ua"], a["va"], ni=ni, nj=nj, nk=nk)
    a["wa"][2 : nk + 1] = rng.uniform(-0.3, 0.3, size=(nk - 1, nj, ni)).astype(np.float32)
    a["uten"][1 : nk + 1, 1 : nj + 1, :] = rng.uniform(-1e-3, 1e-3, size=(nk, nj, ni + 1)).astype(np.float32)
    a["vten"][1 : nk + 1, :, 1 : ni + 1] = rng.uniform(-1e-3, 1e-3, size=(nk, nj + 1, ni)).astype(np.float32)
    a["wten"][2 : nk + 1] = rng.uniform(-1e-2, 1e-2, size=(nk - 1, nj, ni)).astype(np.float32)
    np.copyto(a["u3d"], a["ua"])
    np.copyto(a["v3d"], a["va"])
    np.copyto(a["w3d"], a["wa"])
    np.copyto(a["pp3d"], a["ppi"])
    return a


def make_small(reference: Path) -> None:
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_psolver3_trajectory import (
        TrajectoryAblations,
        cpu_psolver3_trajectory_inplace,
    )
    from cm1core.cuda_sound3_column import sound3_stage_schedule_f32
    from cm1core.cuda_sound3_periodic import cpu_sound3_periodic_three_stage_inplace

    # 1. acoustic operator, three stages, two shapes
    for tag, (ni, nj, nk, seed, dt, nsound) in {
        "sound3_5x4x7": (5, 4, 7, 3, 2.0, 6),
        "sound3_8x6x12": (8, 6, 12, 5, 4.0, 10),
    }.items():
        a = sound_fixture(ni, nj, nk, seed)
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        params = dict(ni=ni, nj=nj, nk=nk, dt=dt, nsound=nsound, rdx=1.0 / 1000.0, rdy=1.0 / 900.0, rdz=1.0 / 450.0)
        result = cpu_sound3_periodic_three_stage_inplace(a, **params)
        outputs = {f"out_{k}": v for k, v in a.items()}
        meta = dict(params, nloop=[s.nloop for s in result.cadence], dts=[s.dts_f32 for s in result.cadence])
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **outputs)
        print("wrote", tag)

    # 2. dry trajectory, two cases, 3 steps each
    for tag, case, steps in (("traj_7x6x7", SMALL_CASE, 3), ("traj_9x5x8", SMALL_CASE_B, 2)):
        a = dry_periodic_state(case)
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        params = dict(ni=case.ni, nj=case.nj, nk=case.nk, dt=case.dt, nsound=case.nsound,
                      dx=case.dx, dy=case.dy, dz=case.dz)
        result = cpu_psolver3_trajectory_inplace(a, steps=steps, **params)
        outputs = {f"out_{k}": v for k, v in a.items()}
        cadence = [
            dict(large_step=c.large_step, nrk=c.nrk, nloop=c.nloop, dts=c.dts_f32, dttmp=c.dttmp_f32,
                 max_tridiagonal_residual=c.max_tridiagonal_residual,
                 horizontal_mass_flux_sum=c.horizontal_mass_flux_sum,
                 total_mass_flux_divergence_sum=c.total_mass_flux_divergence_sum,
                 rigid=c.rigid_w_boundary_exact)
            for c in result.cadence
        ]
        meta = dict(params, steps=steps, cadence=cadence, ledgers=list(result.ledgers))
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **outputs)
        print("wrote", tag)

    # 3. ablations: digests of every array after one step with each term off
    case = SMALL_CASE
    params = dict(ni=case.ni, nj=case.nj, nk=case.nk, dt=case.dt, nsound=case.nsound,
                  dx=case.dx, dy=case.dy, dz=case.dz)
    record = {}
    for bit, field in enumerate(ABLATION_FIELDS):
        a = dry_periodic_state(case)
        cpu_psolver3_trajectory_inplace(a, steps=1, ablations=TrajectoryAblations(**{field: False}), **params)
        record[field] = {"mask": 1 << bit, "digests": {n: digest(a[n]) for n in ALL_ARRAY_NAMES}}
    (HERE / "traj_ablations_7x6x7.json").write_text(json.dumps(record, indent=1, sort_keys=True))
    print("wrote ablations")

    # 4. schedule table
    table = []
    for dt in (0.4, 2.0, 3.0, 5.0, 6.0, 0.6, 1.0, 7.3):
        for nsound in (4, 6, 8, 10, 12, 16):
            for nrk in (1, 2, 3):
                n, d = sound3_stage_schedule_f32(dt, nsound, nrk)
                table.append([dt, nsound, nrk, n, float(np.float32(d))])
    (HERE / "schedule.json").write_text(json.dumps(table))
    print("wrote schedule")


def advection_fixture(ni: int, nj: int, nk: int, seed: int) -> dict[str, np.ndarray]:
    """Padded-lane (ng = 3) inputs of the terrain mass flux and scalar
    advection, with both signs and exact (signed) zeros in every mass flux."""
    ng = 3
    rng = np.random.default_rng(seed)

    def field(shape, lo, hi):
        return rng.uniform(lo, hi, size=shape).astype(np.float32)

    a = {
        "u3d": field((nk + 2, nj + 2 * ng, ni + 1 + 2 * ng), -12.0, 12.0),
        "v3d": field((nk + 2, nj + 1 + 2 * ng, ni + 2 * ng), -12.0, 12.0),
        "w3d": field((nk + 3, nj + 2 * ng, ni + 2 * ng), -3.0, 3.0),
        "rho0_3d": field((nk, nj, ni), 0.6, 1.2),
        "rf0": field((nk + 1, nj, ni), 0.6, 1.2),
        "rgzu": field((nj, ni + 1), 0.95, 1.05),
        "rgzv": field((nj + 1, ni), 0.95, 1.05),
        "dzdx": field((nj, ni), -0.02, 0.02),
        "dzdy": field((nj, ni), -0.02, 0.02),
        "gz": field((nj, ni), 0.97, 1.03),
        "c1": field((nk + 1, nj, ni), 0.3, 0.7),
        "rr0": field((nk, nj, ni), 0.8, 1.6),
        "scalar": field((nk + 2, nj + 2 * ng, ni + 2 * ng), 290.0, 310.0),
        "qscalar": (field((nk + 2, nj + 2 * ng, ni + 2 * ng), 0.0, 1.0) ** 4 * np.float32(0.01)).astype(np.float32),
        "adv_rru": field((nk + 2, nj + 2 * ng, ni + 1 + 2 * ng), -9.0, 9.0),
        "adv_rrv": field((nk + 2, nj + 1 + 2 * ng, ni + 2 * ng), -9.0, 9.0),
        "adv_rrw": field((nk + 3, nj + 2 * ng, ni + 2 * ng), -2.0, 2.0),
        "adv_divx": field((nk, nj, ni), -1e-3, 1e-3),
    }
    a["c2"] = (np.float32(1.0) - a["c1"]).astype(np.float32)
    # smooth stretch of the scalar so WENO weights vary, and flat patches
    a["scalar"][:, :, : ni // 3] = np.float32(300.0)
    for name in ("adv_rru", "adv_rrv", "adv_rrw"):
        flat = a[name].reshape(-1)
        idx = rng.choice(flat.size, size=max(4, flat.size // 25), replace=False)
        flat[idx[: len(idx) // 2]] = np.float32(0.0)
        flat[idx[len(idx) // 2 :]] = np.float32(-0.0)
    # signed zeros on the top interior face where WENO tests rrw > 0
    a["adv_rrw"][nk, ng : ng + 2, ng : ng + 3] = np.float32(-0.0)
    a["adv_rrw"][nk, ng + 2 : ng + 4, ng : ng + 3] = np.float32(0.0)
    return a


def make_advection(reference: Path) -> None:
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_advection5 import cpu_scalar_advection5_inplace, cpu_terrain_mass_flux5_inplace
    from cm1core.cuda_terrain_open_boundary import terrain_static_shapes

    for tag, (ni, nj, nk, seed) in {"adv5_12x10x9": (12, 10, 9, 21), "adv5_9x11x10": (9, 11, 10, 22)}.items():
        a = advection_fixture(ni, nj, nk, seed)
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        outputs = {}
        dx, dy, dz = 1000.0, 900.0, 250.0
        shapes = terrain_static_shapes(ni=ni, nj=nj, nk=nk)
        metrics = {name: np.zeros(shape, dtype=np.float32) for name, shape in shapes.items()}
        for name in ("rho0_3d", "rf0", "rgzu", "rgzv", "dzdx", "dzdy", "gz", "c1", "c2", "rr0"):
            metrics[name][...] = a[name]
        mf = {n: a[n].copy() for n in ("u3d", "v3d", "w3d")}
        for n, src in (("rru", "u3d"), ("rrv", "v3d"), ("rrw", "w3d")):
            mf[n] = np.full_like(a[src], np.float32(7.0))  # untouched words keep this sentinel
        divx = np.full((nk, nj, ni), np.float32(7.0), dtype=np.float32)
        cpu_terrain_mass_flux5_inplace(mf, metrics, divx, ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, dz=dz)
        outputs.update({"out_mf_rru": mf["rru"], "out_mf_rrv": mf["rrv"], "out_mf_rrw": mf["rrw"], "out_mf_divx": divx})
        for nrk in (1, 3):
            for sname, weps in (("scalar", 1.0e-6), ("qscalar", 1.0e-2 * 1.0e-18)):
                arrays = {"rru": a["adv_rru"], "rrv": a["adv_rrv"], "rrw": a["adv_rrw"]}
                fluxes = {"x": np.full_like(a["adv_rru"], np.float32(7.0)),
                          "y": np.full_like(a["adv_rrv"], np.float32(7.0)),
                          "z": np.full_like(a["adv_rrw"], np.float32(7.0))}
                tend = np.full((nk, nj, ni), np.float32(7.0), dtype=np.float32)
                cpu_scalar_advection5_inplace(a[sname], arrays, metrics, a["adv_divx"], tend, fluxes,
                                              ni=ni, nj=nj, nk=nk, nrk=nrk, dx=dx, dy=dy, dz=dz, weps=weps)
                key = f"{sname}_nrk{nrk}"
                outputs.update({f"out_{key}_fx": fluxes["x"], f"out_{key}_fy": fluxes["y"],
                                f"out_{key}_fz": fluxes["z"], f"out_{key}_tend": tend})
        meta = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, dz=dz, weps={"scalar": 1.0e-6, "qscalar": 1.0e-2 * 1.0e-18},
                    sentinel=7.0)
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **outputs)
        print("wrote", tag)


def kessler_fixture(ni: int, nj: int, nk: int, dz: float, seed: int) -> dict[str, np.ndarray]:
    """Compact Kessler driver inputs: a moist, partly saturated column set
    with cloud, rain heavy enough for several fallout sub-steps, and small
    negative mixing ratios for pdefq to repair."""
    rng = np.random.default_rng(seed)
    rd, cp, p00 = 287.04, 1005.7, 1.0e5
    z = (np.arange(nk) + 0.5) * dz
    th0 = 300.0 + 0.004 * z
    pi0 = 1.0 - 9.81 * z / (cp * 305.0)
    shape = (nk, nj, ni)

    def bc(x):
        return np.broadcast_to(x[:, None, None], shape).astype(np.float32).copy()

    a = {
        "ruh": (1.0 + 0.01 * rng.standard_normal(ni)).astype(np.float32),
        "rvh": (1.0 + 0.01 * rng.standard_normal(nj)).astype(np.float32),
        "rmh": (1.0 + 0.02 * rng.random(shape)).astype(np.float32),
        "mh": (1.0 + 0.02 * rng.random(shape)).astype(np.float32),
        "pi0": bc(pi0),
        "th0": bc(th0),
        "th3d": rng.uniform(-1.5, 2.5, shape).astype(np.float32),
        "pp3d": rng.uniform(-2e-4, 2e-4, shape).astype(np.float32),
    }
    t = (a["th0"] + a["th3d"]) * (a["pi0"] + a["pp3d"])
    prs = p00 * (a["pi0"] + a["pp3d"]).astype(np.float64) ** (cp / rd)
    a["prs"] = prs.astype(np.float32)
    a["rho"] = (prs / (rd * t)).astype(np.float32)
    a["rr"] = a["rho"].copy()
    esl = 611.2 * np.exp(17.67 * (t - 273.15) / (t - 29.65))
    qvs = 0.622 * esl / (prs - esl)
    a["qv"] = (qvs * rng.uniform(0.7, 1.08, shape)).astype(np.float32)
    a["qc"] = np.where(rng.random(shape) < 0.5, rng.uniform(0.0, 2.5e-3, shape), 0.0).astype(np.float32)
    a["qr"] = np.where(rng.random(shape) < 0.6, rng.uniform(0.0, 6.0e-3, shape), 0.0).astype(np.float32)
    for name in ("qc", "qr"):
        flat = a[name].reshape(-1)
        idx = rng.choice(flat.size, size=flat.size // 20, replace=False)
        flat[idx] = rng.uniform(-2e-5, 0.0, idx.size).astype(np.float32)
    a["qc"][0, 0, 0] = np.float32(5e-15)  # below rmax: pdefq clears it
    a["fall_velocity"] = np.zeros(shape, np.float32)
    a["rain"] = rng.uniform(0.0, 0.5, (1, nj, ni)).astype(np.float32)
    a["prate"] = np.zeros((nj, ni), np.float32)
    a["asq"] = rng.uniform(-1.0, 1.0, 3)
    a["qbudget"] = rng.uniform(-1.0, 1.0, 10)
    return a


def make_kessler(reference: Path) -> None:
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_gm1_kessler_driver import Gm1KesslerDriverSelection, cpu_gm1_kessler_driver_inplace

    for tag, (ni, nj, nk, dz, dt, eqtset, seed) in {
        "kessler_eqt2_7x5x12": (7, 5, 12, 100.0, 30.0, 2, 31),
        "kessler_eqt1_6x6x10": (6, 6, 10, 150.0, 12.0, 1, 32),
    }.items():
        a = kessler_fixture(ni, nj, nk, dz, seed)
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        result = cpu_gm1_kessler_driver_inplace(a, ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=dz, dt=dt,
                                                selection=Gm1KesslerDriverSelection(equation_set=eqtset))
        outputs = {f"out_{k}": v for k, v in a.items()}
        outputs["out_satadj_iterations"] = result["satadj"]["iterations"]
        meta = dict(ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=dz, dt=dt, eqtset=eqtset,
                    max_fall_substeps=result["max_fall_substeps"])
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **outputs)
        print("wrote", tag, "max nfall", result["max_fall_substeps"],
              "iterations", int(result["satadj"]["iterations"].max()))


APMASSCON_CASES = {
    "apmasscon_9x7x12": (9, 7, 12, 51),
    "apmasscon_13x6x10": (13, 6, 10, 52),
}


def apmasscon_fixture(ni: int, nj: int, nk: int, seed: int) -> dict[str, np.ndarray]:
    """A moist, hydrostatic-looking column set (Exner from 1.0 down to 0.6,
    theta 300-360 K, vapour up to 16 g/kg, moist density from the equation
    of state with a few per-mille of seeded departure) and grid factors near
    1 (ruh, rvh, rmh of a gently stretched grid)."""
    rng = np.random.default_rng(seed)
    f = np.float32
    z = (np.arange(nk) + 0.5) / nk
    pi0 = np.broadcast_to((1.0 - 0.4 * z)[:, None, None], (nk, nj, ni)).astype(f).copy()
    th0 = np.broadcast_to((300.0 + 60.0 * z)[:, None, None], (nk, nj, ni)).astype(f).copy()
    th3d = rng.uniform(-1.5, 2.5, (nk, nj, ni)).astype(f)
    qv = (0.016 * np.exp(-3.0 * z)[:, None, None] * rng.uniform(0.7, 1.0, (nk, nj, ni))).astype(f)
    qv[0, 0, :2] = f(-1.0e-6)  # a negative vapour word takes max(0, qv)
    pp3d = rng.uniform(-2.0e-3, 2.0e-3, (nk, nj, ni)).astype(f)
    pi = (pi0.astype(np.float64) + pp3d)
    prs = (1.0e5 * pi ** (1005.7 / 287.04)).astype(f)
    rho = (prs / ((th0.astype(np.float64) + th3d) * pi * (287.04 + np.maximum(qv, 0.0) * 461.5))
           * rng.uniform(0.997, 1.003, (nk, nj, ni))).astype(f)
    return {"ruh": rng.uniform(0.9, 1.1, ni).astype(f), "rvh": rng.uniform(0.9, 1.1, nj).astype(f),
            "rmh": rng.uniform(0.95, 1.05, (nk, nj, ni)).astype(f), "pi0": pi0, "th0": th0, "th3d": th3d, "qv": qv,
            "pp3d": pp3d, "prs": prs, "rho": rho}


def make_apmasscon(reference: Path) -> None:
    """The final-RK dry-air mass correction through the reference's CPU
    twin: mass1 of a starting state (cpu_initial_dry_mass), then
    cpu_apmasscon_inplace on a state whose dry mass has drifted."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_apmasscon import cpu_apmasscon_inplace, cpu_initial_dry_mass

    for tag, (ni, nj, nk, seed) in APMASSCON_CASES.items():
        start = apmasscon_fixture(ni, nj, nk, seed)
        mass1 = cpu_initial_dry_mass(start, ni=ni, nj=nj, nk=nk)
        a = apmasscon_fixture(ni, nj, nk, seed)
        a["rho"] = (a["rho"] * np.float32(1.0021)).astype(np.float32)  # the drift the correction removes
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        r = cpu_apmasscon_inplace(a, ni=ni, nj=nj, nk=nk, mass1=mass1)
        outputs = {f"out_{k}": a[k] for k in ("pp3d", "prs", "rho")}
        meta = dict(ni=ni, nj=nj, nk=nk, mass1=mass1, mass2=r.mass2_before_f64, pressure_sum=r.pressure_sum_before_f64,
                    correction=r.correction_f32, mass_after=r.mass_after_f64)
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **outputs)
        print("wrote", tag, meta)


KESSLER_LARGE_STEP_CASES = {
    "kessler_large_step_eqt2_7x5x12": (7, 5, 12, 100.0, 30.0, 2, 41),
    "kessler_large_step_eqt1_6x6x10": (6, 6, 10, 150.0, 12.0, 1, 42),
}


def kessler_large_step_fixture(ni: int, nj: int, nk: int, dz: float, seed: int) -> tuple[dict, dict]:
    """Driver inputs plus held-rate carriers of a previous step (small
    seeded rates of the four equation-set-2 fields)."""
    a = kessler_fixture(ni, nj, nk, dz, seed)
    rng = np.random.default_rng(seed + 1000)
    shape = (nk, nj, ni)
    held = {"qpten": rng.normal(0.0, 1e-7, shape).astype(np.float32),
            "qtten": rng.normal(0.0, 2e-3, shape).astype(np.float32),
            "qvten": rng.normal(0.0, 2e-7, shape).astype(np.float32),
            "qcten": rng.normal(0.0, 1e-7, shape).astype(np.float32)}
    return a, held


def make_kessler_large_step(reference: Path) -> None:
    """The once-per-large-step Kessler transition through the reference's CPU
    twin cpu_gm1_kessler_large_step_inplace."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_gm1_kessler_driver import Gm1KesslerDriverSelection
    from cm1core.cuda_gm1_kessler_large_step import cpu_gm1_kessler_large_step_inplace

    for tag, (ni, nj, nk, dz, dt, eqtset, seed) in KESSLER_LARGE_STEP_CASES.items():
        a, held = kessler_large_step_fixture(ni, nj, nk, dz, seed)
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        hin = {f"held_in_{k}": v.copy() for k, v in held.items()}
        result = cpu_gm1_kessler_large_step_inplace(a, held, ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=dz, dt=dt,
                                                    selection=Gm1KesslerDriverSelection(equation_set=eqtset))
        outputs = {f"out_{k}": v for k, v in a.items()}
        hout = {f"held_out_{k}": v for k, v in held.items()}
        meta = dict(ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=dz, dt=dt, eqtset=eqtset,
                    max_fall_substeps=result["driver"]["max_fall_substeps"])
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **hin, **outputs, **hout)
        print("wrote", tag)


def sgs_tke_fixture(ni: int, nj: int, nk: int, seed: int) -> dict[str, np.ndarray]:
    rng = np.random.default_rng(seed)
    cell = (nk + 1, nj, ni)
    a = {
        "ruh": (1.0 + 0.05 * rng.standard_normal(ni)).astype(np.float32),
        "rvh": (1.0 + 0.05 * rng.standard_normal(nj)).astype(np.float32),
        "rmf": rng.uniform(0.7, 1.4, cell).astype(np.float32),
        "nm": rng.uniform(-2e-4, 3e-4, cell).astype(np.float32),
        "defv": rng.uniform(-1e-5, 4e-4, cell).astype(np.float32),
        "defh": rng.uniform(-1e-5, 4e-4, cell).astype(np.float32),
        "tkea": (rng.uniform(0.0, 1.0, cell) ** 3 * 2.5).astype(np.float32),
        "dissten": rng.uniform(-1e-4, 1e-4, cell).astype(np.float32),
    }
    flat = a["tkea"].reshape(-1)
    flat[rng.choice(flat.size, size=flat.size // 10, replace=False)] = np.float32(1e-11)
    for name in ("tk", "grdscl", "rgrdscl", "lenscl", "cme", "ce1", "ce2", "csm", "kmh", "kmv", "khh", "khv",
                 "tketen"):
        a[name] = np.full(cell, np.float32(7.0), dtype=np.float32)
    return a


def make_tke(reference: Path) -> None:
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_sgs_tke import cpu_sgs_tke_inplace, sgs_constants_f32

    for tag, (ni, nj, nk, dx, dy, dz, seed) in {"sgs_tke_9x7x12": (9, 7, 12, 1000.0, 1000.0, 250.0, 41),
                                                 "sgs_tke_6x8x10": (6, 8, 10, 100.0, 120.0, 40.0, 42)}.items():
        a = sgs_tke_fixture(ni, nj, nk, seed)
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        r = cpu_sgs_tke_inplace(a, ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, dz=dz)
        outputs = {f"out_{k}": v for k, v in a.items()}
        meta = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, dz=dz, clipped=r.clipped_tke_words,
                    constants={k: float(v) for k, v in sgs_constants_f32().items()})
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **outputs)
        print("wrote", tag, "clipped", r.clipped_tke_words)


def rk_fixture(ni: int, nj: int, nk: int, seed: int) -> dict[str, np.ndarray]:
    ng = 3
    rng = np.random.default_rng(seed)

    def u(shape, lo, hi):
        return rng.uniform(lo, hi, shape).astype(np.float32)

    cell = (nk, nj, ni)
    a = {
        "th0": u((nk,), 295.0, 340.0),
        "th3d": u(cell, -3.0, 3.0),
        "theta_pad": np.zeros((nk + 2, nj + 2 * ng, ni + 2 * ng), np.float32),
        "theta_a": u(cell, -3.0, 3.0), "theta_held": u(cell, -1e-3, 1e-3), "theta_divterm": u(cell, -1e-3, 1e-3),
        "theta_adv": u(cell, -1e-2, 1e-2),
        "q_a": (u((6,) + cell, 0.0, 1.0) ** 3 * np.float32(0.012)).astype(np.float32),
        "q_held": u((6,) + cell, -1e-6, 1e-6), "q_adv": u((6,) + cell, -2e-5, 2e-5),
        "pd_scalar_a": (u(cell, -0.3, 1.0) * np.float32(2e-3)).astype(np.float32),
        "pd_scalar_padded": (u((nk + 2, nj + 2 * ng, ni + 2 * ng), -0.3, 1.0) * np.float32(2e-3)).astype(np.float32),
        "pd_rho0": u(cell, 0.6, 1.2), "pd_gz": u((nj, ni), 0.97, 1.03),
        "pd_flux_x": u((nk + 2, nj + 2 * ng, ni + 1 + 2 * ng), -8.0, 8.0),
        "pd_flux_y": u((nk + 2, nj + 1 + 2 * ng, ni + 2 * ng), -8.0, 8.0),
        "pd_flux_z": u((nk + 3, nj + 2 * ng, ni + 2 * ng), -2.0, 2.0),
        "pd_directional": u(cell, -4e-6, 4e-6),
    }
    a["q_a"][:, :, 0, :] = np.float32(0.0)
    a["theta_a"][0, 0, :4] = np.float32(1e-31)  # below smeps after the update
    a["pd_rgz"] = (np.float32(1.0) / a["pd_gz"]).astype(np.float32)
    return a


def make_rk(reference: Path) -> None:
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_scalar_moist_rk import (
        cpu_compose_scalar_moist_rk_stage_inplace,
        cpu_pdef_direction_inplace,
        cpu_theta_transport_scalar_inplace,
    )

    for tag, (ni, nj, nk, seed) in {"rk_11x9x8": (11, 9, 8, 51), "rk_7x12x10": (7, 12, 10, 52)}.items():
        a = rk_fixture(ni, nj, nk, seed)
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        out = {}
        pad = a["theta_pad"].copy()
        cpu_theta_transport_scalar_inplace(a["th0"].copy(), a["th3d"].copy(), pad, ni=ni, nj=nj, nk=nk)
        out["out_theta_pad"] = pad
        for nrk in (1, 2, 3):
            tc = np.zeros_like(a["theta_a"])
            qc = np.zeros_like(a["q_a"])
            cpu_compose_scalar_moist_rk_stage_inplace(
                a["theta_a"].copy(), a["q_a"].copy(), a["theta_held"].copy(), a["q_held"].copy(),
                a["theta_divterm"].copy(), a["theta_adv"].copy(), a["q_adv"].copy(), tc, qc, nrk=nrk, dt=5.0)
            out[f"out_theta_cur_{nrk}"] = tc
            out[f"out_q_cur_{nrk}"] = qc
        for axis, spacing in (("x", 1000.0), ("y", 900.0), ("z", 250.0)):
            d = a["pd_directional"].copy()
            cand = np.zeros_like(d)
            cpu_pdef_direction_inplace(a["pd_scalar_a"].copy(), a["pd_scalar_padded"].copy(), a["pd_rho0"].copy(),
                                       a["pd_gz"].copy(), a["pd_rgz"].copy(), a[f"pd_flux_{axis}"].copy(), d, cand,
                                       axis=axis, dt=5.0 / 3.0, spacing=spacing)
            out[f"out_pd_directional_{axis}"] = d
            out[f"out_pd_candidate_{axis}"] = cand
        meta = dict(ni=ni, nj=nj, nk=nk, dt=5.0, pdef_dt=5.0 / 3.0, spacing={"x": 1000.0, "y": 900.0, "z": 250.0})
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **out)
        print("wrote", tag)


def make_bridge(reference: Path) -> None:
    """eqtset=2 stage terms, cell by cell, through the reference's twin."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_moist_stage_bridge import cpu_eqtset2_cell_f32

    rng = np.random.default_rng(61)
    n = 400
    inp = {
        "th0": rng.uniform(295.0, 345.0, n).astype(np.float32),
        "qv0": rng.uniform(0.0, 0.014, n).astype(np.float32),
        "pi0": rng.uniform(0.6, 1.0, n).astype(np.float32),
        "qc0": np.where(rng.random(n) < 0.2, rng.uniform(0.0, 1e-4, n), 0.0).astype(np.float32),
        "qi0": np.where(rng.random(n) < 0.2, rng.uniform(0.0, 1e-4, n), 0.0).astype(np.float32),
        "th3d": rng.uniform(-4.0, 4.0, n).astype(np.float32),
        "pp3d": rng.uniform(-3e-3, 3e-3, n).astype(np.float32),
        "q": rng.uniform(-2e-5, 6e-3, (6, n)).astype(np.float32),
    }
    inp["q"][0] = rng.uniform(-1e-5, 0.016, n).astype(np.float32)
    out = np.zeros((4, n), np.float32)
    for c in range(n):
        r = cpu_eqtset2_cell_f32(th0=inp["th0"][c], qv0=inp["qv0"][c], pi0=inp["pi0"][c], qc0=inp["qc0"][c],
                                 qi0=inp["qi0"][c], th3d=inp["th3d"][c], pp3d=inp["pp3d"][c], qv=inp["q"][0, c],
                                 qc=inp["q"][1, c], qr=inp["q"][2, c], qi=inp["q"][3, c], qs=inp["q"][4, c],
                                 qg=inp["q"][5, c])
        out[:, c] = [r["buoyancy"], r["theta_rho"], r["theta_term"], r["pressure_term"]]
    np.savez_compressed(HERE / "eqtset2_cells.npz", meta=json.dumps({"cells": n}),
                        **{f"in_{k}": v for k, v in inp.items()}, out_terms=out)
    print("wrote eqtset2_cells")


def make_limits(reference: Path) -> None:
    """CM1 limits through the reference's own functions: the small-step
    bound, the diagnostic substep count and the scalar Courant number on a
    table of grids and winds (src/cm1core/gm1_runtime.py:249,284,458), and the
    domain Courant number of advective_courant_number
    (src/cm1core/storm_diagnostics.py:249) run on seeded winds with NumPy in
    place of CuPy (the function only uses cp.add/multiply/sqrt with out=,
    cp.amax, cp.empty and cp.asnumpy)."""
    import contextlib  # noqa: PLC0415
    import types  # noqa: PLC0415

    sys.path.insert(0, str(reference / "src"))
    from cm1core.gm1_runtime import (
        cm1_acoustic_small_step_limit_s,
        cm1_advective_courant,
        cm1_diagnostic_acoustic_substeps,
    )
    from cm1core.storm_diagnostics import advective_courant_number

    rng = np.random.default_rng(71)
    table = []
    for dx, dy in ((1000.0, 1000.0), (250.0, 250.0), (333.33, 500.0), (2000.0, 1500.0), (100.0, 3000.0),
                   (20.0, 20.0)):
        for dt in (1.0, 2.5, 6.0, 7.5, 10.0, 12.0, 30.0):
            u, v, w = (float(x) for x in rng.normal(0.0, 25.0, 3))
            dz = float(rng.uniform(20.0, 500.0))
            table.append({
                "dx": dx, "dy": dy, "dt": dt, "dz": dz, "u": u, "v": v, "w": w,
                "limit": cm1_acoustic_small_step_limit_s(dx_m=dx, dy_m=dy),
                "nsound": cm1_diagnostic_acoustic_substeps(dt_s=dt, dx_m=dx, dy_m=dy),
                "courant": cm1_advective_courant(dt_s=dt, dx_m=dx, dy_m=dy, dz_m=dz, u_m_s=u, v_m_s=v, w_m_s=w),
            })

    shim = types.SimpleNamespace(float32=np.float32, empty=np.empty, add=np.add, multiply=np.multiply,
                                 sqrt=np.sqrt, amax=np.amax, asnumpy=np.asarray)
    cases = {}
    for tag, (nx, ny, nz, dx, dy, dz, dt, stretch, poison) in {
        "a": (12, 10, 9, 1000.0, 1000.0, 500.0, 6.0, False, None),
        "b": (9, 11, 6, 250.0, 333.0, 100.0, 2.0, True, None),
        "c": (16, 8, 7, 500.0, 500.0, 250.0, 3.0, False, (0, "nan")),
        "d": (10, 10, 8, 1000.0, 1000.0, 500.0, 6.0, True, (3, "nan")),
        "e": (8, 9, 5, 1000.0, 1000.0, 500.0, 6.0, False, (2, "inf")),
    }.items():
        u = rng.normal(5.0, 20.0, (nz, ny, nx + 1)).astype(np.float32)
        v = rng.normal(-3.0, 15.0, (nz, ny + 1, nx)).astype(np.float32)
        w = rng.normal(0.0, 8.0, (nz + 1, ny, nx)).astype(np.float32)
        uh = np.ones(nx + 6, np.float32)
        vh = np.ones(ny + 6, np.float32)
        mh = np.ones(nz, np.float32)
        if stretch:
            uh[3:3 + nx] = rng.uniform(0.8, 1.25, nx).astype(np.float32)
            vh[3:3 + ny] = rng.uniform(0.8, 1.25, ny).astype(np.float32)
            mh[:] = rng.uniform(0.5, 2.0, nz).astype(np.float32)
        if poison is not None:
            level, kind = poison
            u[level, ny // 2, nx // 2] = np.float32("nan") if kind == "nan" else np.float32("inf")
        grid = types.SimpleNamespace(nx=nx, ny=ny, nz=nz, dx_m=dx, dy_m=dy, dz_m=dz)
        runtime = types.SimpleNamespace(
            cp=shim, stream=contextlib.nullcontext(),
            config=types.SimpleNamespace(grid=grid, dt_s=dt),
            dynamics=types.SimpleNamespace(fields={"u3d": u, "v3d": v, "w3d": w}, arrays={"uh": uh, "vh": vh},
                                           metrics={"mh": mh}))
        with np.errstate(invalid="ignore", over="ignore"):
            number = advective_courant_number(runtime)
        cases[tag] = dict(meta=json.dumps({"nx": nx, "ny": ny, "nz": nz, "dx": dx, "dy": dy, "dz": dz, "dt": dt,
                                           "courant": number}),
                          u=u, v=v, w=w, uh=uh[3:3 + nx].copy(), vh=vh[3:3 + ny].copy(), mh=mh)
    np.savez_compressed(HERE / "limits_courant.npz",
                        table=json.dumps(table),
                        **{f"{tag}_{k}": val for tag, c in cases.items() for k, val in c.items()})
    print("wrote limits_courant", {t: json.loads(c["meta"])["courant"] for t, c in cases.items()})


def deformation_fixture(ni: int, nj: int, nk: int, seed: int) -> dict[str, np.ndarray]:
    """Terrain-following calcdef inputs: a smooth seeded terrain, its CM1
    metric terms, sheared winds with noise, a decreasing density."""
    rng = np.random.default_rng(seed)
    f = np.float32
    dx, dy, dz = f(100.0), f(120.0), f(200.0)
    zt = f(nk) * dz
    jj, ii = np.meshgrid(np.arange(nj), np.arange(ni), indexing="ij")
    zs = (150.0 + 60.0 * np.sin(0.7 * ii + 0.3) * np.cos(0.5 * jj) + rng.uniform(0, 10, (nj, ni))).astype(f)
    a = {"gz": (zt / (zt - zs)).astype(f), "rgz": ((zt - zs) / zt).astype(f)}
    zu = np.empty((nj, ni + 1), f)
    for i in range(ni + 1):
        zu[:, i] = f(0.5) * (zs[:, max(i - 1, 0)] + zs[:, min(i, ni - 1)])
    zv = np.empty((nj + 1, ni), f)
    for j in range(nj + 1):
        zv[j] = f(0.5) * (zs[max(j - 1, 0)] + zs[min(j, nj - 1)])
    a["rgzu"] = ((zt - zu) / zt).astype(f)
    a["rgzv"] = ((zt - zv) / zt).astype(f)
    a["gzu"] = (zt / (zt - zu)).astype(f)
    a["gzv"] = (zt / (zt - zv)).astype(f)
    sigf = (np.arange(nk + 1, dtype=f) * dz)[:, None, None]
    a["gx"] = ((zt - sigf) * a["gz"] * (a["rgzu"][:, 1:] - a["rgzu"][:, :-1]) / dx).astype(f)
    a["gy"] = ((zt - sigf) * a["gz"] * (a["rgzv"][1:] - a["rgzv"][:-1]) / dy).astype(f)
    k = np.arange(nk)[:, None, None]
    a["u3d"] = (5.0 + 0.4 * k + rng.normal(0, 1.5, (nk, nj, ni + 1))).astype(f)
    a["v3d"] = (-2.0 + 0.3 * k + rng.normal(0, 1.5, (nk, nj + 1, ni))).astype(f)
    w = rng.normal(0, 0.8, (nk + 1, nj, ni)).astype(f)
    w[0] = 0.0
    w[nk] = 0.0
    a["w3d"] = w
    rho = (1.15 * np.exp(-0.00011 * (k + 0.5) * 200.0) + rng.uniform(-0.01, 0.01, (nk, nj, ni))).astype(f)
    a["rho"] = rho
    rf = np.empty((nk + 1, nj, ni), f)
    rf[1:nk] = f(0.5) * (rho[:-1] + rho[1:])
    rf[0] = f(1.5) * rho[0] - f(0.5) * rho[1]
    rf[nk] = f(1.5) * rho[nk - 1] - f(0.5) * rho[nk - 2]
    a["rf"] = rf
    c1 = rng.uniform(0.4, 0.6, (nk + 1, nj, ni)).astype(f)
    a["c1"] = c1
    a["c2"] = (f(1.0) - c1).astype(f)
    a["defv"] = np.full((nk + 1, nj, ni), np.nan, f)
    a["defh"] = np.full((nk + 1, nj, ni), np.nan, f)
    return {n: np.ascontiguousarray(v) for n, v in a.items()} | {"_spacing": np.array([dx, dy, dz], f)}


def moist_nm_fixture(ni: int, nj: int, nk: int, seed: int) -> dict[str, np.ndarray]:
    """calcnm inputs whose temperatures span ~300 K to ~210 K, with vapour
    near saturation and seeded condensate, so the liquid, mixed-phase and ice
    branches all occur."""
    rng = np.random.default_rng(seed)
    f = np.float32
    z = (np.arange(nk) + 0.5) / nk
    t_col = 300.0 - 95.0 * z
    pi0 = (1.0 - 0.45 * z).astype(f)
    th0 = (t_col / pi0).astype(f)
    cells = (nk, nj, ni)
    a = {"pi0": pi0, "th0": th0}
    a["pp3d"] = rng.normal(0, 2e-4, cells).astype(f)
    a["th3d"] = rng.normal(0, 1.5, cells).astype(f)
    exner = pi0[:, None, None] + a["pp3d"]
    a["prs"] = (1.0e5 * exner.astype(np.float64) ** (1005.7 / 287.04)).astype(f)
    temp = (th0[:, None, None] + a["th3d"]) * exner
    es = 611.2 * np.exp(17.67 * (temp - 273.15) / (temp - 29.65))
    qsat = 0.622 * es / (a["prs"] - es)
    q = np.zeros((6,) + cells, f)
    q[0] = (qsat * rng.uniform(0.85, 1.1, cells)).astype(f)
    for s, scale in ((1, 4e-4), (2, 2e-4), (3, 2e-4), (4, 1e-4), (5, 1e-4)):
        q[s] = np.where(rng.random(cells) < 0.5, rng.uniform(0, scale, cells), 0.0).astype(f)
    a["q3d"] = q
    face = (nk + 1, nj, ni)
    c1 = rng.uniform(0.4, 0.6, face).astype(f)
    a["c1"] = c1
    a["c2"] = (f(1.0) - c1).astype(f)
    a["mf"] = rng.uniform(0.9, 1.1, face).astype(f)
    for n in ("nm",):
        a[n] = np.full(face, np.nan, f)
    for n in ("temperature", "qt", "thv", "qvci"):
        a[n] = np.full(cells, np.nan, f)
    a["saturation_mask"] = np.full(cells, 7, np.uint8)
    return {n: np.ascontiguousarray(v) for n, v in a.items()}


def make_closure(reference: Path) -> None:
    """calcdef and calcnm through the reference's CPU twins on seeded inputs."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_moist_nm import cpu_moist_nm_inplace
    from cm1core.cuda_terrain_deformation import cpu_terrain_deformation_inplace

    for tag, (ni, nj, nk, seed) in {"calcdef_9x7x8": (9, 7, 8, 41), "calcdef_12x6x10": (12, 6, 10, 43)}.items():
        a = deformation_fixture(ni, nj, nk, seed)
        dx, dy, dz = (float(x) for x in a.pop("_spacing"))
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        cpu_terrain_deformation_inplace(a, ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, dz=dz)
        meta = {"ni": ni, "nj": nj, "nk": nk, "dx": dx, "dy": dy, "dz": dz}
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs,
                            out_defv=a["defv"], out_defh=a["defh"])
        print("wrote", tag)
    for tag, (ni, nj, nk, seed) in {"moist_nm_8x6x14": (8, 6, 14, 47), "moist_nm_5x9x20": (5, 9, 20, 53)}.items():
        a = moist_nm_fixture(ni, nj, nk, seed)
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        r = cpu_moist_nm_inplace(a, ni=ni, nj=nj, nk=nk, dz=250.0)
        meta = {"ni": ni, "nj": nj, "nk": nk, "dz": 250.0, "saturated": r.saturated_words, "liquid": r.liquid_words,
                "mixed": r.mixed_words, "ice": r.ice_words}
        outs = {f"out_{k}": a[k] for k in ("nm", "temperature", "qt", "thv", "qvci", "saturation_mask")}
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **outs)
        print("wrote", tag, meta)


def tke_evolution_fixture(ni: int, nj: int, nk: int, seed: int) -> dict[str, np.ndarray]:
    """Seeded inputs of the terrain-lane TKE evolution: positive TKE and
    eddy viscosities, a terrain metric, mass fluxes of both signs."""
    rng = np.random.default_rng(seed)
    f = np.float32
    face, mass = (nk + 1, nj, ni), (nk, nj, ni)
    ng = 3
    a = {
        "tke3d": rng.uniform(0.0, 2.0, face).astype(f), "tkea": rng.uniform(0.0, 2.0, face).astype(f),
        "tketen": rng.normal(0.0, 1e-3, face).astype(f), "kmh": rng.uniform(1.0, 60.0, face).astype(f),
        "kmv": rng.uniform(1.0, 40.0, face).astype(f), "rho": rng.uniform(0.7, 1.2, mass).astype(f),
        "rf": rng.uniform(0.7, 1.2, face).astype(f), "mh": rng.uniform(0.9, 1.1, mass).astype(f),
        "mf": rng.uniform(0.9, 1.1, face).astype(f), "gz": rng.uniform(1.0, 1.05, (nj, ni)).astype(f),
        "rgzu": rng.uniform(0.95, 1.0, (nj, ni + 1)).astype(f), "rgzv": rng.uniform(0.95, 1.0, (nj + 1, ni)).astype(f),
        "c1": rng.uniform(0.4, 0.6, face).astype(f), "rrf0": rng.uniform(0.8, 1.4, face).astype(f),
        "rru": rng.normal(4.0, 8.0, (nk + 2, nj + 2 * ng, ni + 1 + 2 * ng)).astype(f),
        "rrv": rng.normal(-2.0, 8.0, (nk + 2, nj + 1 + 2 * ng, ni + 2 * ng)).astype(f),
        "rrw": rng.normal(0.0, 1.5, (nk + 3, nj + 2 * ng, ni + 2 * ng)).astype(f),
        "divx": rng.normal(0.0, 1e-3, mass).astype(f),
    }
    a["rgz"] = (f(1.0) / a["gz"]).astype(f)
    a["c2"] = (f(1.0) - a["c1"]).astype(f)
    for k in (0, nk):
        a["tke3d"][k] = 0.0
        a["tkea"][k] = 0.0
    return {n: np.ascontiguousarray(v) for n, v in a.items()}


def make_tke_evolution(reference: Path) -> None:
    """turbt + three TKE RK stages through the reference's CPU twin."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_tke_evolution import cpu_tke_evolution_inplace

    for tag, (ni, nj, nk, seed) in {"tke_evolution_9x8x10": (9, 8, 10, 71), "tke_evolution_7x10x9": (7, 10, 9, 73)}.items():
        a = tke_evolution_fixture(ni, nj, nk, seed)
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        p = {"ni": ni, "nj": nj, "nk": nk, "dx": 250.0, "dy": 300.0, "dz": 200.0, "dt": 3.0}
        r = cpu_tke_evolution_inplace(a, **p)
        meta = dict(p, stage_sha256=r["stage_sha256"])
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs,
                            **{f"out_{k}": a[k] for k in ("tke3d", "tkea", "tketen")})
        print("wrote", tag)


def momentum_fixture(ni: int, nj: int, nk: int, seed: int) -> tuple[dict[str, np.ndarray], dict[str, np.ndarray],
                                                                    np.ndarray]:
    """Padded-lane momentum-advection inputs: seeded winds with filled halos,
    accumulated tendencies, terrain metrics."""
    rng = np.random.default_rng(seed)
    f = np.float32
    ng = 3
    su, sv, sw = (nk + 2, nj + 2 * ng, ni + 1 + 2 * ng), (nk + 2, nj + 1 + 2 * ng, ni + 2 * ng), \
        (nk + 3, nj + 2 * ng, ni + 2 * ng)
    a = {
        "u3d": rng.normal(6.0, 6.0, su).astype(f), "uten": rng.normal(0.0, 1e-3, su).astype(f),
        "rru": np.zeros(su, f), "v3d": rng.normal(-2.0, 6.0, sv).astype(f),
        "vten": rng.normal(0.0, 1e-3, sv).astype(f), "rrv": np.zeros(sv, f),
        "w3d": rng.normal(0.0, 1.5, sw).astype(f), "wten": rng.normal(0.0, 1e-3, sw).astype(f),
        "rrw": np.zeros(sw, f), "uh": rng.uniform(0.95, 1.05, ni + 2 * ng).astype(f),
        "vh": rng.uniform(0.95, 1.05, nj + 2 * ng).astype(f),
    }
    face = (nk + 1, nj, ni)
    m = {
        "rho0_3d": rng.uniform(0.7, 1.2, (nk, nj, ni)).astype(f), "rf0": rng.uniform(0.7, 1.2, face).astype(f),
        "c2": rng.uniform(0.4, 0.6, face).astype(f), "gz": rng.uniform(1.0, 1.05, (nj, ni)).astype(f),
        "gzu": rng.uniform(1.0, 1.05, (nj, ni + 1)).astype(f), "gzv": rng.uniform(1.0, 1.05, (nj + 1, ni)).astype(f),
        "dzdx": rng.normal(0.0, 0.02, (nj, ni)).astype(f), "dzdy": rng.normal(0.0, 0.02, (nj, ni)).astype(f),
    }
    m["rrf0"] = (f(1.0) / m["rf0"]).astype(f)
    m["rgzu"] = (f(1.0) / m["gzu"]).astype(f)
    m["rgzv"] = (f(1.0) / m["gzv"]).astype(f)
    m["c1"] = (f(1.0) - m["c2"]).astype(f)
    m["rr0"] = (f(1.0) / m["rho0_3d"]).astype(f)
    return a, m, np.zeros((nk, nj, ni), f)


MOMENTUM_CASES = {
    "momentum5_open_9x8x10": (9, 8, 10, 81, (2, 2, 2, 2)),
    "momentum5_perx_8x9x9": (8, 9, 9, 83, (1, 1, 2, 2)),
    "momentum5_walls_10x7x8": (10, 7, 8, 89, (3, 4, 1, 1)),
}


def make_momentum(reference: Path) -> None:
    """Terrain/open momentum advection through the reference's CPU twin."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_momentum_advection5 import cpu_terrain_open_momentum_advection5_inplace
    from cm1core.cuda_terrain_open_boundary import terrain_static_shapes

    for tag, (ni, nj, nk, seed, sides) in MOMENTUM_CASES.items():
        a, m, divx = momentum_fixture(ni, nj, nk, seed)
        full = {n: np.zeros(shape, np.float32) for n, shape in terrain_static_shapes(ni=ni, nj=nj, nk=nk).items()}
        full.update(m)
        inputs = {f"in_{k}": v.copy() for k, v in {**a, **m}.items()}
        p = {"ni": ni, "nj": nj, "nk": nk, "dx": 400.0, "dy": 350.0, "dz": 180.0}
        cpu_terrain_open_momentum_advection5_inplace(a, full, divx, nrk=1, lateral_sides=sides, **p)
        meta = dict(p, lateral_sides=list(sides))
        outs = {f"out_{k}": a[k] for k in ("uten", "vten", "wten", "rru", "rrv", "rrw")}
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **outs, out_divx=divx)
        print("wrote", tag)


TERRAIN_OPEN_ARRAYS = ("ppi", "pp3d", "ppx", "ppd", "piadv", "ppterm", "ppten", "thv", "qk", "pk1", "pk2", "mm",
                       "fpk", "divh", "hadvp", "dum3", "elim_c", "elim_d", "tri_aa", "tri_bb", "tri_cc", "tri_dd",
                       "tri_pivot", "tri_residual", "ua", "u3d", "uten", "rru", "va", "v3d", "vten", "rrv", "wa",
                       "w3d", "wten", "rrw", "radbcw", "radbce", "radbcs", "radbcn", "uh", "vh", "ruf", "rvf",
                       "scalar")


def terrain_open_fixture(ni: int, nj: int, nk: int, seed: int) -> tuple[dict[str, np.ndarray],
                                                                       dict[str, np.ndarray]]:
    """Seeded terrain/open acoustic-stage inputs: winds, pressure family and
    radiation histories with random halos, garbage in every scratch array
    (the stage must overwrite or zero it), and the 25 terrain metrics with a
    non-broadcast base density."""
    rng = np.random.default_rng(seed)
    f = np.float32
    ng = 3
    pr, su, sv = (nk + 2, nj + 2, ni + 2), (nk + 2, nj + 2 * ng, ni + 1 + 2 * ng), (nk + 2, nj + 1 + 2 * ng, ni + 2 * ng)
    sw, ss = (nk + 3, nj + 2 * ng, ni + 2 * ng), (nk + 2, nj + 2 * ng, ni + 2 * ng)
    a: dict[str, np.ndarray] = {}
    for n in TERRAIN_OPEN_ARRAYS[:24]:
        a[n] = rng.normal(0.0, 0.5, pr).astype(f)
    pert = rng.normal(0.0, 2e-4, pr).astype(f)
    a["ppi"] = pert.copy()
    a["pp3d"] = (pert + rng.normal(0.0, 2e-5, pr)).astype(f)
    a["ppx"] = (pert + rng.normal(0.0, 2e-5, pr)).astype(f)
    a["piadv"] = (f(0.9) + rng.normal(0.0, 2e-3, pr)).astype(f)
    a["ppterm"] = (a["piadv"] * f(287.04 / (1005.7 - 287.04))).astype(f)
    a["thv"] = (f(300.0) + np.arange(nk + 2, dtype=f)[:, None, None] * f(0.4) + rng.normal(0.0, 0.3, pr)).astype(f)
    a["ppten"] = rng.normal(0.0, 1e-6, pr).astype(f)
    a["u3d"] = rng.normal(8.0, 3.0, su).astype(f)
    a["ua"] = (a["u3d"] + rng.normal(0.0, 0.05, su)).astype(f)
    a["uten"] = rng.normal(0.0, 2e-3, su).astype(f)
    a["rru"] = rng.normal(0.0, 1.0, su).astype(f)
    a["v3d"] = rng.normal(-3.0, 3.0, sv).astype(f)
    a["va"] = (a["v3d"] + rng.normal(0.0, 0.05, sv)).astype(f)
    a["vten"] = rng.normal(0.0, 2e-3, sv).astype(f)
    a["rrv"] = rng.normal(0.0, 1.0, sv).astype(f)
    a["w3d"] = rng.normal(0.0, 0.5, sw).astype(f)
    a["wa"] = (a["w3d"] + rng.normal(0.0, 0.02, sw)).astype(f)
    a["wten"] = rng.normal(0.0, 2e-3, sw).astype(f)
    a["rrw"] = rng.normal(0.0, 1.0, sw).astype(f)
    a["radbcw"] = rng.uniform(-25.0, 0.0, (nk + 2, nj + 2 * ng)).astype(f)
    a["radbce"] = rng.uniform(0.0, 25.0, (nk + 2, nj + 2 * ng)).astype(f)
    a["radbcs"] = rng.uniform(-25.0, 0.0, (nk + 2, ni + 2 * ng)).astype(f)
    a["radbcn"] = rng.uniform(0.0, 25.0, (nk + 2, ni + 2 * ng)).astype(f)
    a["uh"] = np.ones(ni + 2 * ng, f)
    a["vh"] = np.ones(nj + 2 * ng, f)
    a["ruf"] = np.ones(ni + 1 + 2 * ng, f)
    a["rvf"] = np.ones(nj + 1 + 2 * ng, f)
    a["scalar"] = rng.normal(1.0, 0.2, ss).astype(f)
    mass, face, plane = (nk, nj, ni), (nk + 1, nj, ni), (nj, ni)
    m: dict[str, np.ndarray] = {}
    terrain = rng.uniform(0.0, 400.0, plane).astype(f)
    m["terrain_msl"] = terrain
    m["zh"] = rng.uniform(100.0, 9000.0, mass).astype(f)
    m["zf"] = rng.uniform(0.0, 9000.0, face).astype(f)
    for n, shape in (("mh", mass), ("mf", face)):
        m[n] = rng.uniform(0.95, 1.05, shape).astype(f)
        m["r" + n] = (f(1.0) / m[n]).astype(f)
    m["c1"] = rng.uniform(0.4, 0.6, face).astype(f)
    m["c2"] = (f(1.0) - m["c1"]).astype(f)
    base = np.linspace(1.15, 0.6, nk, dtype=f)
    m["rho0_3d"] = (base[:, None, None] * rng.uniform(0.98, 1.02, mass)).astype(f)
    m["rr0"] = (f(1.0) / m["rho0_3d"]).astype(f)
    m["rf0"] = (np.linspace(1.18, 0.58, nk + 1, dtype=f)[:, None, None] * rng.uniform(0.98, 1.02, face)).astype(f)
    m["rrf0"] = (f(1.0) / m["rf0"]).astype(f)
    for n, shape in (("gz", plane), ("gzu", (nj, ni + 1)), ("gzv", (nj + 1, ni))):
        m[n] = rng.uniform(1.0, 1.06, shape).astype(f)
    m["rgz"] = (f(1.0) / m["gz"]).astype(f)
    m["rgzu"] = (f(1.0) / m["gzu"]).astype(f)
    m["rgzv"] = (f(1.0) / m["gzv"]).astype(f)
    m["dzdx"] = rng.normal(0.0, 0.02, plane).astype(f)
    m["dzdy"] = rng.normal(0.0, 0.02, plane).astype(f)
    m["gx"] = rng.normal(0.0, 0.005, face).astype(f)
    m["gxu"] = rng.normal(0.0, 0.005, (nk + 1, nj, ni + 1)).astype(f)
    m["gy"] = rng.normal(0.0, 0.005, face).astype(f)
    m["gyv"] = rng.normal(0.0, 0.005, (nk + 1, nj + 1, ni)).astype(f)
    return a, m


TERRAIN_OPEN_CASES = {
    # name: (ni, nj, nk, seed, dt, nsound, dx, dy, dz)
    "tos_seeded_9x7x8": (9, 7, 8, 97, 3.0, 6, 500.0, 400.0, 333.3),
    "tos_seeded_6x10x6": (6, 10, 6, 101, 2.4, 8, 300.0, 350.0, 180.0),
}
TERRAIN_OPEN_ABLATIONS = ("open_consumption", "terrain_pressure_gradient", "transformed_divergence",
                          "pressure_advection", "implicit_vertical_solve", "between_step_pressure_fill",
                          "radiation_history_production", "stage_family_fills")


def make_terrain_open(reference: Path) -> None:
    """The terrain/open acoustic stage through the reference's CPU twin:
    the reference test's own 5x4x5 inputs and two seeded cases over three RK
    stages (full arrays and per-stage digests of every array), each of the
    eight ablations, and non-default alph/kdiv."""
    sys.path.insert(0, str(reference / "src"))
    sys.path.insert(0, str(reference / "tests"))
    from cm1core.cuda_psolver3_terrain_open import TerrainOpenSoundAblations, cpu_psolver3_terrain_open_stage_inplace
    import test_cuda_psolver3_terrain_open as reftest

    def run(a, m, p, *, ablations=None, alph=None, kdiv=None):
        stages = []
        for nrk in (1, 2, 3):
            d = cpu_psolver3_terrain_open_stage_inplace(a, m, nrk=nrk, ablations=ablations, alph=alph, kdiv=kdiv, **p)
            stages.append({"nrk": nrk, "nloop": d.nloop, "dts_f32": d.dts_f32,
                           "max_tridiagonal_residual": d.max_tridiagonal_residual,
                           "digests": {n: digest(a[n]) for n in TERRAIN_OPEN_ARRAYS}})
        return stages

    cases = {"tos_reftest_5x4x5": (reftest._arrays(5, 4, 5), reftest._metrics(5, 4, 5),
                                   dict(ni=5, nj=4, nk=5, dt=0.6, nsound=6, dx=100.0, dy=100.0, dz=200.0))}
    for tag, (ni, nj, nk, seed, dt, nsound, dx, dy, dz) in TERRAIN_OPEN_CASES.items():
        a, m = terrain_open_fixture(ni, nj, nk, seed)
        cases[tag] = (a, m, dict(ni=ni, nj=nj, nk=nk, dt=dt, nsound=nsound, dx=dx, dy=dy, dz=dz))
    for tag, (a, m, p) in cases.items():
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        minputs = {f"metric_{k}": v for k, v in m.items()}
        t0 = time.time()
        stages = run(a, m, p)
        meta = dict(p, stages=stages)
        if tag == "tos_reftest_5x4x5":
            abl = {}
            for name in TERRAIN_OPEN_ABLATIONS:
                b = {k[3:]: v.copy() for k, v in inputs.items()}
                run(b, m, p, ablations=TerrainOpenSoundAblations(**{name: False}))
                abl[name] = {n: digest(b[n]) for n in TERRAIN_OPEN_ARRAYS}
            meta["ablations"] = abl
        if tag == "tos_seeded_9x7x8":
            b = {k[3:]: v.copy() for k, v in inputs.items()}
            meta["alph_kdiv"] = {"alph": 0.5, "kdiv": 0.05, "stages": run(b, m, p, alph=0.5, kdiv=0.05)}
        outs = {f"out_{k}": a[k] for k in TERRAIN_OPEN_ARRAYS}
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **minputs, **outs)
        print("wrote", tag, round(time.time() - t0, 1), "s", flush=True)


def moist_piece_fixture(ni: int, nj: int, nk: int, seed: int) -> dict[str, np.ndarray]:
    """Seeded inputs of the moist-step pieces: padded winds / mass fluxes,
    a moisture field near zero with some negative words (so the pdef repair
    rows fire), buoyancy on the scalar layout, terrain metrics."""
    rng = np.random.default_rng(seed)
    f = np.float32
    su, sv, sw = (nk + 2, nj + 6, ni + 7), (nk + 2, nj + 7, ni + 6), (nk + 3, nj + 6, ni + 6)
    ss, mass, face = (nk + 2, nj + 6, ni + 6), (nk, nj, ni), (nk + 1, nj, ni)
    a = {
        "rru": rng.normal(0.0, 8.0, su).astype(f), "rrv": rng.normal(0.0, 8.0, sv).astype(f),
        "rrw": rng.normal(0.0, 1.0, sw).astype(f), "uten": rng.normal(0.0, 1e-3, su).astype(f),
        "vten": rng.normal(0.0, 1e-3, sv).astype(f), "wten": rng.normal(0.0, 1e-3, sw).astype(f),
        "dum8": rng.normal(0.0, 0.05, ss).astype(f), "thterm": rng.uniform(80.0, 120.0, mass).astype(f),
        "scalar_padded": np.where(rng.random(ss) < 0.15, rng.normal(-2e-6, 1e-6, ss),
                                  rng.uniform(0.0, 1.2e-2, ss)).astype(f),
        "scalar_a": rng.uniform(0.0, 1.2e-2, mass).astype(f),
        "c1": rng.uniform(0.4, 0.6, face).astype(f), "rho0_3d": rng.uniform(0.6, 1.2, mass).astype(f),
        "rf0": rng.uniform(0.6, 1.2, face).astype(f), "gz": rng.uniform(0.97, 1.03, (nj, ni)).astype(f),
        "rgzu": rng.uniform(0.95, 1.05, (nj, ni + 1)).astype(f), "rgzv": rng.uniform(0.95, 1.05, (nj + 1, ni)).astype(f),
        "dzdx": rng.normal(0.0, 0.02, (nj, ni)).astype(f), "dzdy": rng.normal(0.0, 0.02, (nj, ni)).astype(f),
        "gxu": rng.normal(0.0, 0.004, (nk + 1, nj, ni + 1)).astype(f),
        "gyv": rng.normal(0.0, 0.004, (nk + 1, nj + 1, ni)).astype(f),
        "divx": rng.normal(0.0, 1e-3, mass).astype(f),
    }
    a["c2"] = (f(1.0) - a["c1"]).astype(f)
    a["rgz"] = (f(1.0) / a["gz"]).astype(f)
    a["rr0"] = (f(1.0) / a["rho0_3d"]).astype(f)
    return a


def make_fills(reference: Path) -> None:
    """The open-lateral fills through the reference's own functions on seeded
    arrays with garbage halos."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_sound3_open_boundary import (cpu_bcp_open_inplace, cpu_bcs_open_inplace, cpu_bcu_open_inplace,
                                                   cpu_bcv_open_inplace, cpu_bcw_open_inplace)

    ni, nj, nk = 9, 7, 6
    rng = np.random.default_rng(321)
    shapes = {"pressure": (nk + 2, nj + 2, ni + 2), "scalar": (nk + 2, nj + 6, ni + 6), "u": (nk + 2, nj + 6, ni + 7),
              "v": (nk + 2, nj + 7, ni + 6), "w": (nk + 3, nj + 6, ni + 6), "w_keep_ends": (nk + 3, nj + 6, ni + 6)}
    out = {}
    for kind, shape in shapes.items():
        q = rng.normal(0.0, 1.0, shape).astype(np.float32)
        out[f"in_{kind}"] = q.copy()
        if kind == "pressure":
            cpu_bcp_open_inplace(q, ni=ni, nj=nj, nk=nk)
        elif kind == "scalar":
            cpu_bcs_open_inplace(q, ni=ni, nj=nj, nk=nk)
        elif kind == "u":
            cpu_bcu_open_inplace(q, ni=ni, nj=nj, nk=nk)
        elif kind == "v":
            cpu_bcv_open_inplace(q, ni=ni, nj=nj, nk=nk)
        else:
            cpu_bcw_open_inplace(q, ni=ni, nj=nj, nk=nk, flag=1 if kind == "w" else 0)
        out[f"out_{kind}"] = q
    np.savez_compressed(HERE / "open_fills_9x7x6.npz", meta=json.dumps(dict(ni=ni, nj=nj, nk=nk)), **out)
    print("wrote open_fills_9x7x6")


def make_wk(reference: Path) -> None:
    """CM1 r21.1's own Weisman-Klemp base state (isnd=5, nz=40, dz=500 m) as
    float32 words, from the CM1 output the reference keeps
    (tests/data/cm1-ref-24x24/stats-run-t1500.npz: th0, qv0, pi0, prs0;
    variants.json: the derived variant's pi0 column), plus the sealed SHA-256
    digests of the qv0 and pi0 words in the reference's binary32 restatement
    tests (rust/cm1-state/src/storm_initialization.rs, test
    hydrostatic_fixed_point_is_settled_at_the_source_iteration_count)."""
    import re  # noqa: PLC0415

    data = reference / "tests" / "data" / "cm1-ref-24x24"
    state = np.load(data / "stats-run-t1500.npz")
    variants = json.loads((data / "variants.json").read_text())
    words = {n: [f"{int(w):08x}" for w in state[n].astype(np.float32).view(np.uint32)]
             for n in ("th0", "qv0", "pi0", "prs0")}
    column = variants["variants"]["derived"]["block"]["pi0_column"]
    rust = (reference / "rust" / "cm1-state" / "src" / "storm_initialization.rs").read_text()
    sealed = dict(re.findall(r'raw_sha256\(twenty\.(qv_kg_per_kg|pi)\(\)\),\s*"([0-9a-f]{64})"', rust))
    record = {
        "case": "CM1 r21.1 supercell namelist, isnd=5 imoist=1, nz=40, dz=500 m (mass heights 250..19750 m)",
        "nz": 40, "dz": 500.0,
        "cm1_words": words,
        "cm1_pi0_column_derived_variant": column,
        "sealed_sha256": {"qv0": sealed["qv_kg_per_kg"], "pi0": sealed["pi"]},
    }
    (HERE / "wk_cm1_nz40.json").write_text(json.dumps(record, indent=1, sort_keys=True))
    print("wrote wk_cm1_nz40")


def make_c1(reference: Path, checkpoints: list[int]) -> None:
    """Digests after each checkpoint N, each from a fresh state with one call
    of steps=N (the reference refuses a non-fresh entry state, ppx != pp3d,
    src/cm1core/cuda_psolver3_trajectory.py:242-246).  Checkpoints already in
    the output file are kept."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_psolver3_trajectory import cpu_psolver3_trajectory_inplace

    case = DRY_BUBBLE_64
    out = HERE / "traj_c1_digests.json"
    fresh = dry_periodic_state(case)
    record = json.loads(out.read_text()) if out.exists() else {}
    record["case"] = "dry bubble 64x64x40 (dx=dy=1 km, dz=500 m, dt=6 s, nsound=6)"
    record["input_digests"] = {n: digest(fresh[n]) for n in ALL_ARRAY_NAMES}
    record.setdefault("steps", {})
    params = dict(ni=case.ni, nj=case.nj, nk=case.nk, dt=case.dt, nsound=case.nsound,
                  dx=case.dx, dy=case.dy, dz=case.dz)
    for n in checkpoints:
        if str(n) in record["steps"]:
            continue
        a = copy.deepcopy(fresh)
        t0 = time.time()
        result = cpu_psolver3_trajectory_inplace(a, steps=n, **params)
        record["steps"][str(n)] = {
            "digests": {name: digest(a[name]) for name in ALL_ARRAY_NAMES},
            "max_abs": {name: float(np.max(np.abs(a[name]))) for name in ("u3d", "v3d", "w3d", "pp3d", "th3d")},
            "max_tridiagonal_residual": max(c.max_tridiagonal_residual for c in result.cadence),
            "reference_cpu_seconds": time.time() - t0,
        }
        out.write_text(json.dumps(record, indent=1, sort_keys=True))
        print("checkpoint", n, time.time() - t0, flush=True)


VERTICAL_CASES = {
    # name: (stretch_z, nk, dz, ztop, str_bot, str_top, dz_bot, dz_top)
    "child_15km_nk75": (1, 75, 100.0, 15000.0, 200.0, 7000.0, 20.0, 320.0),
    "stretch_20_500_nk80": (1, 80, 100.0, 20800.0, 200.0, 15800.0, 20.0, 500.0),
    "stretch_from_ground_nk50": (1, 50, 200.0, 11500.0, 0.0, 8000.0, 50.0, 350.0),
    "uniform_nk80_dz250": (0, 80, 250.0, 20000.0, 0.0, 0.0, 0.0, 0.0),
    "uniform_nk40_dz500": (0, 40, 500.0, 20000.0, 0.0, 0.0, 0.0, 0.0),
}
VERTICAL_REFUSALS = {
    "infeasible_dz_bot": (1, 75, 100.0, 15000.0, 200.0, 7000.0, 30.0, 320.0),
    "uniform_wrong_top": (0, 40, 500.0, 19000.0, 0.0, 0.0, 0.0, 0.0),
    "stretch_z2": (2, 75, 200.0, 15000.0, 0.0, 0.0, 0.0, 0.0),
    "too_few_levels": (0, 3, 500.0, 1500.0, 0.0, 0.0, 0.0, 0.0),
}


def make_vertical(reference: Path) -> None:
    """CM1 vertical coordinates (stretch_z 0 and 1) through the reference's
    own build_vertical_levels and derive_stretch_z1: every profile's float32
    words, rds/rdsf, the Fornberg weights, the derived segment counts and the
    sealed digests; refused parameter sets with the reference's error."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cm1_vertical_grid import build_vertical_levels
    from cm1core.cuda_stretch_z1 import StretchZ1Parameters, derive_stretch_z1

    def words(a) -> list[int]:
        return [int(w) for w in np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)]

    out = {"cases": {}, "refusals": {}}
    for name, (sz, nk, dz, ztop, sb, st, db, dt) in VERTICAL_CASES.items():
        lv = build_vertical_levels(stretch_z=sz, nk=nk, dz_m=dz, ztop_m=ztop, str_bot_m=sb, str_top_m=st,
                                   dz_bot_m=db, dz_top_m=dt)
        rec = {"args": [sz, nk, dz, ztop, sb, st, db, dt], "ztop_m": lv.ztop_m, "sha256": lv.sha256,
               "cgs": words(np.array(lv.cgs, np.float32)), "cgt": words(np.array(lv.cgt, np.float32))}
        for f in ("zf", "zh", "sigmaf", "sigma", "mh", "mf", "rmh", "rmf", "rds", "rdsf"):
            rec[f] = words(getattr(lv, f))
        p = lv.stretch_parameters()
        d = derive_stretch_z1(p)
        rec["derived"] = {"nk1": d.nk1, "nk2": d.nk2, "nk3": d.nk3,
                          "nominal": words(np.array([d.nominal_dz_f32], np.float32))[0],
                          "c1": words(np.array([d.c1_f32], np.float32))[0],
                          "c2": words(np.array([d.c2_f32], np.float32))[0]}
        rec["stretch_parameters"] = [p.nk, p.dz, p.ztop, p.str_bot, p.str_top, p.dz_bot, p.dz_top]
        out["cases"][name] = rec
    for name, (sz, nk, dz, ztop, sb, st, db, dt) in VERTICAL_REFUSALS.items():
        try:
            build_vertical_levels(stretch_z=sz, nk=nk, dz_m=dz, ztop_m=ztop, str_bot_m=sb, str_top_m=st,
                                  dz_bot_m=db, dz_top_m=dt)
        except Exception as e:  # noqa: BLE001 - the reference's refusal is the record
            out["refusals"][name] = {"args": [sz, nk, dz, ztop, sb, st, db, dt], "error": type(e).__name__,
                                     "message": str(e)[:200]}
        else:
            raise AssertionError(f"{name} was not refused by the reference")
    from cm1core.stretch_z1_child_15km import STRETCH_Z1_CHILD_15KM_PROFILE_SHA256

    out["sealed_child_15km_profile_sha256"] = dict(STRETCH_Z1_CHILD_15KM_PROFILE_SHA256)
    (HERE / "vertical_levels.json").write_text(json.dumps(out, indent=1, sort_keys=True))


WARM_RAIN_CASES = {"warm_rain_8x6x5": (8, 6, 5, 20.0, 51), "warm_rain_7x9x6": (7, 9, 6, 6.0, 52)}


def warm_rain_fixture(ni: int, nj: int, nk: int, seed: int, saturation: tuple[float, float]) -> dict[str, np.ndarray]:
    """Compact Kessler inputs for the collection and single-pass adjustment
    pins: qv at saturation * U(saturation), cloud water on both sides of the
    autoconversion threshold 0.001 and some cells without, rain from none to
    heavy enough for the qc limiter."""
    rng = np.random.default_rng(seed)
    rd, cp, p00, dz = 287.04, 1005.7, 1.0e5, 400.0
    z = (np.arange(nk) + 0.5) * dz
    shape = (nk, nj, ni)

    def bc(x):
        return np.broadcast_to(x[:, None, None], shape).astype(np.float32).copy()

    a = {
        "ruh": (1.0 + 0.01 * rng.standard_normal(ni)).astype(np.float32),
        "rvh": (1.0 + 0.01 * rng.standard_normal(nj)).astype(np.float32),
        "rmh": (1.0 + 0.02 * rng.random(shape)).astype(np.float32),
        "pi0": bc(1.0 - 9.81 * z / (cp * 302.0)),
        "th0": bc(300.0 + 0.004 * z),
        "th3d": rng.uniform(-1.5, 2.5, shape).astype(np.float32),
        "pp3d": rng.uniform(-2e-4, 2e-4, shape).astype(np.float32),
    }
    t = (a["th0"] + a["th3d"]) * (a["pi0"] + a["pp3d"])
    prs = p00 * (a["pi0"] + a["pp3d"]).astype(np.float64) ** (cp / rd)
    a["prs"] = prs.astype(np.float32)
    a["rho"] = (prs / (rd * t)).astype(np.float32)
    a["rr"] = a["rho"].copy()
    esl = 611.2 * np.exp(17.67 * (t - 273.15) / (t - 29.65))
    qvs = 0.622 * esl / (prs - esl)
    a["qv"] = (qvs * rng.uniform(*saturation, shape)).astype(np.float32)
    u = rng.random(shape)
    a["qc"] = np.where(u < 0.2, 0.0, np.where(u < 0.6, rng.uniform(1e-5, 9.5e-4, shape),
                                              rng.uniform(1.05e-3, 3e-3, shape))).astype(np.float32)
    u = rng.random(shape)
    a["qr"] = np.where(u < 0.3, 0.0, np.where(u < 0.8, rng.uniform(1e-6, 2e-3, shape),
                                              rng.uniform(8e-3, 2e-2, shape))).astype(np.float32)
    return a


def make_warm_rain(reference: Path) -> None:
    """The two Kessler pieces the adjoint differentiates, through the
    reference's own CPU code: cpu_gm1_kessler_local_inplace on supersaturated
    cells (no rain evaporation, so its qc and qr are the collection's), and
    the driver's _cpu_satadj with equation set 1 on cells from 85% to 115% of
    saturation."""
    sys.path.insert(0, str(reference / "src"))
    import cm1core.cuda_gm1_kessler_driver as drv
    from cm1core.cuda_gm1_kessler_local import cpu_gm1_kessler_local_inplace

    for tag, (ni, nj, nk, dt, seed) in WARM_RAIN_CASES.items():
        a = warm_rain_fixture(ni, nj, nk, seed, (1.01, 1.2))
        a["budget"] = np.zeros(3, np.float64)
        inputs = {f"in_coll_{k}": v.copy() for k, v in a.items()}
        cpu_gm1_kessler_local_inplace(a, ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=400.0, dt=dt)
        outputs = {f"out_coll_{k}": a[k].copy() for k in ("qv", "qc", "qr", "th3d")}
        b = warm_rain_fixture(ni, nj, nk, seed + 100, (0.85, 1.15))
        b["qbudget"] = np.zeros(10, np.float64)
        inputs.update({f"in_sat_{k}": v.copy() for k, v in b.items()})
        drv._cpu_satadj(np, b, ni=ni, nj=nj, nk=nk, dx=np.float32(1000.0), dy=np.float32(1000.0),
                        dz=np.float32(400.0), dt=np.float32(dt), equation_set=1)
        outputs.update({f"out_sat_{k}": b[k].copy() for k in ("th3d", "qv", "qc", "rho")})
        meta = dict(ni=ni, nj=nj, nk=nk, dt=dt)
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **outputs)
        print("wrote", tag)


# (ni, nj, nk, seed, level_uniform): level_uniform cases hold kmh/kmv
# constant on each level and s12's edge corners equal to the nearest
# interior corner (the flat calcdef's own edge rule), so the flat column's
# gettau/turbu texts and this terrain twin form the same sums
STRESS_CASES = {"stress_7x6x5": (7, 6, 5, 61, False), "stress_9x8x7": (9, 8, 7, 62, True)}


def stress_fixture(ni: int, nj: int, nk: int, seed: int, level_uniform: bool = False) -> dict[str, np.ndarray]:
    """Seeded inputs of the SGS stress: strains and eddy coefficients of
    both signs and magnitudes, positive densities and column metrics, flat
    terrain (gz = rgz = 1, zero slopes)."""
    from oracle.stress import stress_shapes

    rng = np.random.default_rng(seed)
    sh = stress_shapes(ni, nj, nk)
    f = np.float32
    a = {}
    for n in ("s11", "s22", "s33", "s12", "s13", "s23", "u3d", "v3d", "w3d"):
        a[n] = rng.normal(0.0, 0.3, sh[n]).astype(f)
    for n in ("kmh", "kmv"):
        a[n] = rng.uniform(0.5, 40.0, sh[n]).astype(f)
        if level_uniform:
            a[n][:] = a[n][:, :1, :1]
    if level_uniform:
        jj = np.clip(np.arange(nj + 1), 1, nj - 1)
        ii = np.clip(np.arange(ni + 1), 1, ni - 1)
        a["s12"] = np.ascontiguousarray(a["s12"][:, jj][:, :, ii])
    a["rho"] = rng.uniform(0.4, 1.2, sh["rho"]).astype(f)
    a["rf"] = rng.uniform(0.4, 1.2, sh["rf"]).astype(f)
    a["mh"] = rng.uniform(0.7, 1.4, sh["mh"]).astype(f)
    a["mf"] = rng.uniform(0.7, 1.4, sh["mf"]).astype(f)
    for n, s in (("gz", (nj, ni)), ("rgz", (nj, ni)), ("gzu", (nj, ni + 1)), ("rgzu", (nj, ni + 1)),
                 ("gzv", (nj + 1, ni)), ("rgzv", (nj + 1, ni))):
        a[n] = np.ones(s, f)
    a["gxu"] = np.zeros((nk + 1, nj, ni + 1), f)
    a["gyv"] = np.zeros((nk + 1, nj + 1, ni), f)
    for n in ("t11", "t22", "t33", "t12", "t13", "t23"):
        a[n] = np.zeros(sh[n], f)
    for n in ("uten", "vten", "wten"):
        a[n] = rng.normal(0.0, 1.0e-3, sh[n]).astype(f)
    return a


def make_stress(reference: Path) -> None:
    """gettau and turbu/turbv/turbw through the reference's CPU twin
    cpu_sgs_stress_tendency_inplace (src/cm1core/cuda_sgs_stress_tendency.py:292)
    on seeded strains and coefficients, square 100 m grid, flat terrain."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_sgs_stress_tendency import cpu_sgs_stress_tendency_inplace

    for tag, (ni, nj, nk, seed, level_uniform) in STRESS_CASES.items():
        a = stress_fixture(ni, nj, nk, seed, level_uniform)
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        cpu_sgs_stress_tendency_inplace(a, ni=ni, nj=nj, nk=nk, dx=100.0, dy=100.0, dz=50.0, dt=0.6)
        outputs = {f"out_{k}": a[k].copy() for k in ("t11", "t22", "t33", "t12", "t13", "t23", "uten", "vten",
                                                     "wten")}
        meta = dict(ni=ni, nj=nj, nk=nk, dx=100.0, dy=100.0, dz=50.0, dt=0.6, level_uniform=level_uniform)
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **outputs)
        print("wrote", tag)


# (ni, nj, nk, seed): dx = dy = 128 m, so every product with 1/dx is exact
# and the terrain twin's fluxes on flat metrics form the flat text's words
TURBS_CASES = {"turbs_8x7x6": (8, 7, 6, 71), "turbs_11x9x10": (11, 9, 10, 72)}


def turbs_fixture(ni: int, nj: int, nk: int, seed: int) -> dict[str, np.ndarray]:
    """Seeded inputs of turbs: theta and six moisture rows with horizontal
    and vertical structure, positive diffusivities, densities and column
    metrics, flat terrain."""
    rng = np.random.default_rng(seed)
    f = np.float32
    mass, face = (nk, nj, ni), (nk + 1, nj, ni)
    a = {"th0": np.linspace(300.0, 340.0, nk).astype(f), "tha": rng.normal(0.0, 1.5, mass).astype(f),
         "qa": np.abs(rng.normal(0.0, 4.0e-3, (6, nk, nj, ni))).astype(f),
         "rho": rng.uniform(0.4, 1.2, mass).astype(f)}
    a["rr"] = (f(1.0) / a["rho"]).astype(f)
    a["rf"] = rng.uniform(0.4, 1.2, face).astype(f)
    a["mh"] = rng.uniform(0.7, 1.4, mass).astype(f)
    a["mf"] = rng.uniform(0.7, 1.4, face).astype(f)
    a["khh"] = rng.uniform(0.5, 80.0, face).astype(f)
    a["khv"] = rng.uniform(0.5, 80.0, face).astype(f)
    for n, s in (("gz", (nj, ni)), ("rgz", (nj, ni)), ("rgzu", (nj, ni + 1)), ("rgzv", (nj + 1, ni))):
        a[n] = np.ones(s, f)
    for n, s in (("gx", face), ("gxu", (nk + 1, nj, ni + 1)), ("gy", face), ("gyv", (nk + 1, nj + 1, ni))):
        a[n] = np.zeros(s, f)
    a["thten1"] = rng.normal(0.0, 1.0e-3, mass).astype(f)
    a["qten"] = rng.normal(0.0, 1.0e-6, (6, nk, nj, ni)).astype(f)
    return a


def make_turbs(reference: Path) -> None:
    """turbs for theta and the six moisture rows through the reference's
    CPU twin cpu_gm1_scalar_turbulence_inplace
    (src/cm1core/cuda_gm1_scalar_turbulence.py:414) on flat metrics."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_gm1_scalar_turbulence import cpu_gm1_scalar_turbulence_inplace

    for tag, (ni, nj, nk, seed) in TURBS_CASES.items():
        a = turbs_fixture(ni, nj, nk, seed)
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        cpu_gm1_scalar_turbulence_inplace(a, ni=ni, nj=nj, nk=nk, dx=128.0, dy=128.0, dz=40.0, dt=0.6)
        outputs = {f"out_{k}": a[k].copy() for k in ("thten1", "qten")}
        meta = dict(ni=ni, nj=nj, nk=nk, dx=128.0, dy=128.0, dz=40.0, dt=0.6)
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), **inputs, **outputs)
        print("wrote", tag)


# (ni, nj, nk, seed): the reference's sealed damping selection (irdamp 1,
# 15 km top, damping from 12 km, rdalpha 1/300) on a uniform 200 m column
RAYLEIGH_CASES = {"rayleigh_9x7x75": (9, 7, 75, 81), "rayleigh_6x8x75": (6, 8, 75, 82)}


def make_rayleigh(reference: Path) -> None:
    """The damping coefficients and the held tendencies through the
    reference's own CPU code: cpu_build_rayleigh_coefficients on the one-halo
    heights of a uniform 200 m, 75-level column, and cpu_rayleigh_held_inplace
    (src/cm1core/cuda_rayleigh_held.py:213, :264) on seeded winds and theta."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.cuda_rayleigh_held import cpu_build_rayleigh_coefficients, cpu_rayleigh_held_inplace

    f = np.float32
    for tag, (ni, nj, nk, seed) in RAYLEIGH_CASES.items():
        rng = np.random.default_rng(seed)
        zf1 = (np.arange(nk + 1) * 200.0).astype(f)
        zh1 = ((np.arange(nk) + 0.5) * 200.0).astype(f)
        zh = np.ascontiguousarray(np.broadcast_to(zh1[:, None, None], (nk, nj + 2, ni + 2)))
        zf = np.ascontiguousarray(np.broadcast_to(zf1[:, None, None], (nk + 1, nj + 2, ni + 2)))
        co = cpu_build_rayleigh_coefficients(zh, zf)
        a = {"tauh": co.tauh, "taus": co.taus, "tauf": co.tauf,
             "u0": rng.normal(5.0, 8.0, nk).astype(f), "v0": rng.normal(0.0, 4.0, nk).astype(f),
             "ua": rng.normal(6.0, 9.0, (nk, nj, ni + 1)).astype(f),
             "va": rng.normal(0.0, 5.0, (nk, nj + 1, ni)).astype(f),
             "wa": rng.normal(0.0, 2.0, (nk, nj, ni)).astype(f), "tha": rng.normal(0.0, 2.0, (nk, nj, ni)).astype(f),
             "uten1": np.zeros((nk, nj, ni + 1), f), "vten1": np.zeros((nk, nj + 1, ni), f),
             "wten1": np.zeros((nk, nj, ni), f), "thten1": np.zeros((nk, nj, ni), f)}
        inputs = {f"in_{k}": v.copy() for k, v in a.items()}
        cpu_rayleigh_held_inplace(a, ni=ni, nj=nj, nk=nk)
        outputs = {f"out_{k}": a[k].copy() for k in ("uten1", "vten1", "wten1", "thten1")}
        meta = dict(ni=ni, nj=nj, nk=nk, dz=200.0, damping_start_m=12000.0, rdalpha=0.0033333333333)
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(meta), zh=zh1, zf=zf1, **inputs, **outputs)
        print("wrote", tag)


IDISS_CASES = {"idiss_7x6x9": (7, 6, 9, 91)}


def make_idiss(reference: Path) -> None:
    """The dissipative heating cell by cell through the reference's own
    scalar mirror cpu_idiss_cell_f32 (src/cm1core/eqtset2_energy_terms.py:176)
    on seeded dissipation rates, pressures and six moisture rows."""
    sys.path.insert(0, str(reference / "src"))
    from cm1core.eqtset2_energy_terms import cpu_idiss_cell_f32

    f = np.float32
    for tag, (ni, nj, nk, seed) in IDISS_CASES.items():
        rng = np.random.default_rng(seed)
        a = {"dissten": rng.uniform(0.0, 0.05, (nk + 1, nj, ni)).astype(f),
             "pi0": np.linspace(1.0, 0.55, nk).astype(f), "ppi": rng.normal(0.0, 2e-3, (nk, nj, ni)).astype(f),
             "qa": np.abs(rng.normal(0.0, 3e-3, (6, nk, nj, ni))).astype(f),
             "thten1": rng.normal(0.0, 1e-3, (nk, nj, ni)).astype(f)}
        out = a["thten1"].copy()
        for k in range(nk):
            for j in range(nj):
                for i in range(ni):
                    q = a["qa"][:, k, j, i]
                    r = cpu_idiss_cell_f32(thten1=float(out[k, j, i]), dissten_lower=float(a["dissten"][k, j, i]),
                                           dissten_upper=float(a["dissten"][k + 1, j, i]), pi0=float(a["pi0"][k]),
                                           ppi=float(a["ppi"][k, j, i]), qv=float(q[0]), qc=float(q[1]),
                                           qr=float(q[2]), qi=float(q[3]), qs=float(q[4]), qg=float(q[5]))
                    out[k, j, i] = r["thten1"]
        np.savez_compressed(HERE / f"{tag}.npz", meta=json.dumps(dict(ni=ni, nj=nj, nk=nk)),
                            **{f"in_{k}": v for k, v in a.items()}, out_thten1=out)
        print("wrote", tag)


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--reference", type=Path, required=True, help="root of the reference source tree")
    p.add_argument("what", choices=("small", "c1", "advection", "kessler", "tke", "rk", "bridge", "wk", "limits", "closure", "tkeevo", "momentum", "terrainopen", "kesslerstep", "fills", "vertical", "warmrain", "apmasscon", "stress", "turbs", "rayleigh", "idiss"))
    p.add_argument("--checkpoints", type=int, nargs="+", default=[1])
    args = p.parse_args()
    if args.what == "small":
        make_small(args.reference)
    elif args.what == "advection":
        make_advection(args.reference)
    elif args.what == "kessler":
        make_kessler(args.reference)
    elif args.what == "rk":
        make_rk(args.reference)
    elif args.what == "bridge":
        make_bridge(args.reference)
    elif args.what == "tke":
        make_tke(args.reference)
    elif args.what == "wk":
        make_wk(args.reference)
    elif args.what == "limits":
        make_limits(args.reference)
    elif args.what == "closure":
        make_closure(args.reference)
    elif args.what == "tkeevo":
        make_tke_evolution(args.reference)
    elif args.what == "momentum":
        make_momentum(args.reference)
    elif args.what == "terrainopen":
        make_terrain_open(args.reference)
    elif args.what == "kesslerstep":
        make_kessler_large_step(args.reference)
    elif args.what == "fills":
        make_fills(args.reference)
    elif args.what == "warmrain":
        make_warm_rain(args.reference)
    elif args.what == "vertical":
        make_vertical(args.reference)
    elif args.what == "apmasscon":
        make_apmasscon(args.reference)
    elif args.what == "stress":
        make_stress(args.reference)
    elif args.what == "turbs":
        make_turbs(args.reference)
    elif args.what == "rayleigh":
        make_rayleigh(args.reference)
    elif args.what == "idiss":
        make_idiss(args.reference)
    else:
        make_c1(args.reference, sorted(set(args.checkpoints)))


if __name__ == "__main__":
    main()
