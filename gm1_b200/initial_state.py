"""Seeded synthetic initial states for the serial-periodic dry lane.

The dry warm bubble of the 64x64x40 benchmark case: a neutral theta0 = 300 K
base state in CM1's discrete hydrostatic form, a cos^2 warm bubble (CM1
iinit=1, init3d.F:450-482 as restated in
rust/cm1-state/src/initial_perturbation.rs:449-466) plus seeded uniform noise,
and every carrier laid out in the padded shapes of the reference operator API
with the contract its trajectory launcher checks
(src/cm1core/cuda_psolver3_trajectory.py:162-247): horizontally uniform
profiles, c1 + c2 == 1, periodic halos, rigid w faces, current == A carriers
and ppx == pp3d.

The base state follows CM1's discrete hydrostatic recursion (base.F:415-418 as
restated in rust/cm1-state/src/storm_initialization.rs:265-270) with the dry
equation of state; ghost levels copy the nearest interior level.  The base
state is an input: parity is checked on identical inputs, so these choices do
not enter any parity claim.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .arrays import (
    default_periodic_face_weights,
    fill_periodic_scalar_inplace,
    fill_periodic_uv_inplace,
    trajectory_array_shapes,
)

G = 9.81
RD = 287.04
CP = 1005.7
P00 = 1.0e5


@dataclass(frozen=True)
class DryBubbleCase:
    """Parameters of one dry periodic warm-bubble case."""

    ni: int = 64
    nj: int = 64
    nk: int = 40
    dx: float = 1000.0
    dy: float = 1000.0
    dz: float = 500.0
    dt: float = 6.0
    nsound: int = 6
    steps: int = 10
    theta0: float = 300.0
    surface_pressure: float = 1.0e5
    bubble_amplitude: float = 2.0
    bubble_radius_h: float = 10_000.0
    bubble_radius_v: float = 1_500.0
    bubble_center_z: float = 1_500.0
    noise_amplitude: float = 0.01
    seed: int = 1
    # optional background wind and a seeded smooth perturbation of u, v, w
    # (zero in the benchmark case; small fixtures use it to drive both
    # upwind branches of every flux)
    u0: float = 0.0
    v0: float = 0.0
    wind_perturbation: float = 0.0

    @property
    def cells(self) -> int:
        return self.ni * self.nj * self.nk


# The 64x64x40 dry bubble: dx = dy = 1 km, dz = 500 m, dt = 6 s, 6 acoustic
# substeps, 10 large steps, +2 K bubble (r_h 10 km, r_v 1.5 km, z_c 1.5 km)
# with +/-0.01 K noise from numpy.random.default_rng(1).
DRY_BUBBLE_64 = DryBubbleCase()


def _base_profiles(case: DryBubbleCase) -> dict[str, np.ndarray]:
    nk, dz = case.nk, case.dz
    zh = (np.arange(1, nk + 1, dtype=np.float64) - 0.5) * dz
    th = np.full(nk, case.theta0, dtype=np.float64)
    pi_sfc = (case.surface_pressure / P00) ** (RD / CP)
    pi = np.empty(nk, dtype=np.float64)
    pi[0] = pi_sfc - G * zh[0] / (CP * 0.5 * (case.theta0 + th[0]))
    for k in range(1, nk):
        pi[k] = pi[k - 1] - G * (zh[k] - zh[k - 1]) / (CP * 0.5 * (th[k] + th[k - 1]))
    prs = P00 * pi ** (CP / RD)
    rho = prs / (RD * th * pi)
    rho_sfc = case.surface_pressure / (RD * case.theta0 * pi_sfc)

    def padded(interior: np.ndarray) -> np.ndarray:
        out = np.empty(nk + 2, dtype=np.float64)
        out[1 : nk + 1] = interior
        out[0] = interior[0]
        out[nk + 1] = interior[-1]
        return out

    th0 = padded(th).astype(np.float32)
    pi0 = padded(pi).astype(np.float32)
    rho0 = padded(rho).astype(np.float32)
    # face density rf0(k) on the face below mass level k: the c1/c2 blend of
    # the two neighbouring levels (uniform grid: c1 = c2 = 1/2), the surface
    # density at k = 1 and a linear extrapolation at the lid.
    rf = np.empty(nk + 2, dtype=np.float64)
    rf[2 : nk + 1] = 0.5 * (rho[:-1] + rho[1:])
    rf[1] = rho_sfc
    rf[nk + 1] = 1.5 * rho[-1] - 0.5 * rho[-2]
    rf[0] = rf[1]
    rf0 = rf.astype(np.float32)
    one = np.float32(1.0)
    return {
        "th0": th0,
        "pi0": pi0,
        "rho0": rho0,
        "rf0": rf0,
        "rr0": (one / rho0).astype(np.float32),
        "rrf0": (one / rf0).astype(np.float32),
        "rth0": (one / th0).astype(np.float32),
        "c1": np.full(nk + 2, 0.5, dtype=np.float32),
        "c2": np.full(nk + 2, 0.5, dtype=np.float32),
        "mh": np.ones(nk + 2, dtype=np.float32),
        "mf": np.ones(nk + 2, dtype=np.float32),
    }


def _bubble(case: DryBubbleCase) -> np.ndarray:
    ni, nj, nk = case.ni, case.nj, case.nk
    xh = (np.arange(1, ni + 1, dtype=np.float64) - 0.5) * case.dx
    yh = (np.arange(1, nj + 1, dtype=np.float64) - 0.5) * case.dy
    zh = (np.arange(1, nk + 1, dtype=np.float64) - 0.5) * case.dz
    xc = 0.5 * ni * case.dx
    yc = 0.5 * nj * case.dy
    rx = (xh[None, None, :] - xc) / case.bubble_radius_h
    ry = (yh[None, :, None] - yc) / case.bubble_radius_h
    rz = (zh[:, None, None] - case.bubble_center_z) / case.bubble_radius_v
    beta = np.sqrt(rx * rx + ry * ry + rz * rz)
    return np.where(beta < 1.0, case.bubble_amplitude * np.cos(0.5 * np.pi * beta) ** 2, 0.0)


def dry_periodic_state(case: DryBubbleCase = DRY_BUBBLE_64) -> dict[str, np.ndarray]:
    """Every array of the dry trajectory for ``case`` as float32 host arrays."""

    ni, nj, nk = case.ni, case.nj, case.nk
    shapes = trajectory_array_shapes(ni, nj, nk)
    a = {name: np.zeros(shape, dtype=np.float32) for name, shape in shapes.items()}
    a["dtu0"], a["dtv0"] = default_periodic_face_weights(ni, nj)
    for name in ("uf", "vf", "uh", "vh"):
        a[name].fill(np.float32(1.0))
    for name, profile in _base_profiles(case).items():
        a[name][...] = profile[:, None, None]

    rng = np.random.default_rng(case.seed)
    noise = rng.uniform(-case.noise_amplitude, case.noise_amplitude, size=(nk, nj, ni))
    a["th3d"][1 : nk + 1, 1 : nj + 1, 1 : ni + 1] = (_bubble(case) + noise).astype(np.float32)
    fill_periodic_scalar_inplace(a["th3d"], ni=ni, nj=nj, nk=nk)

    if case.u0 or case.v0 or case.wind_perturbation:
        amp = case.wind_perturbation
        wr = np.random.default_rng(case.seed + 1000)
        phase = wr.uniform(0.0, 2.0 * np.pi, size=6)
        zf = np.arange(nk, dtype=np.float64) / max(nk - 1, 1)
        for k in range(nk):
            f = np.arange(ni + 1, dtype=np.float64)
            j = np.arange(nj, dtype=np.float64)
            xu = 2.0 * np.pi * f / ni
            yu = 2.0 * np.pi * (j + 0.5) / nj
            u = case.u0 + amp * np.sin(xu[None, :] + phase[0]) * np.cos(yu[:, None] + phase[1]) * (
                1.0 + 0.5 * zf[k]
            )
            a["u3d"][k + 1, 1 : nj + 1, :] = u.astype(np.float32)
            g = np.arange(nj + 1, dtype=np.float64)
            i = np.arange(ni, dtype=np.float64)
            xv = 2.0 * np.pi * (i + 0.5) / ni
            yv = 2.0 * np.pi * g / nj
            v = case.v0 + amp * np.cos(xv[None, :] + phase[2]) * np.sin(yv[:, None] + phase[3]) * (
                1.0 - 0.3 * zf[k]
            )
            a["v3d"][k + 1, :, 1 : ni + 1] = v.astype(np.float32)
        # the duplicate periodic faces must be bit-identical
        a["u3d"][1 : nk + 1, 1 : nj + 1, ni] = a["u3d"][1 : nk + 1, 1 : nj + 1, 0]
        a["v3d"][1 : nk + 1, nj, 1 : ni + 1] = a["v3d"][1 : nk + 1, 0, 1 : ni + 1]
        for q in range(2, nk + 1):
            z = np.sin(np.pi * (q - 1) / nk)
            i = np.arange(ni, dtype=np.float64)
            j = np.arange(nj, dtype=np.float64)
            w = 0.1 * amp * z * np.sin(2.0 * np.pi * i[None, :] / ni + phase[4]) * np.sin(
                2.0 * np.pi * j[:, None] / nj + phase[5]
            )
            a["w3d"][q] = w.astype(np.float32)
        fill_periodic_uv_inplace(a["u3d"], a["v3d"], ni=ni, nj=nj, nk=nk)

    for cur, carrier in (("u3d", "ua"), ("v3d", "va"), ("w3d", "wa"), ("pp3d", "ppi"), ("th3d", "tha")):
        np.copyto(a[carrier], a[cur])
    np.copyto(a["ppx"], a["pp3d"])
    return a
