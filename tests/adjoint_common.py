"""A seeded warm-rain transport case for the adjoint tests: frozen open-sided
mass fluxes of both signs, column metrics, a moist state around saturation
with cloud on both sides of the autoconversion threshold and rain from none
to heavy (numpy float32, host)."""

from __future__ import annotations

import numpy as np

NG = 3


def warm_rain_case(ni=16, nj=12, nk=10, seed=3, dx=1000.0, dy=1000.0, dz=400.0):
    rng = np.random.default_rng(seed)
    rd, cp, p00 = 287.04, 1005.7, 1.0e5
    f32 = np.float32

    def smooth(shape, amp, base=0.0):
        # a few random Fourier modes plus noise, so both flux signs occur
        z, y, x = np.meshgrid(*[np.linspace(0, 2 * np.pi, n) for n in shape], indexing="ij")
        out = np.full(shape, base, np.float64)
        for _ in range(4):
            kz, ky, kx = rng.integers(1, 3, 3)
            out += amp * rng.uniform(0.3, 1.0) * np.sin(kz * z + rng.uniform(0, 6)) * np.sin(ky * y + rng.uniform(0, 6)) \
                * np.cos(kx * x + rng.uniform(0, 6))
        out += 0.1 * amp * rng.standard_normal(shape)
        return out.astype(f32)

    frozen = {
        "rru": smooth((nk + 2, nj + 2 * NG, ni + 1 + 2 * NG), 8.0, 2.0),
        "rrv": smooth((nk + 2, nj + 1 + 2 * NG, ni + 2 * NG), 8.0, -1.0),
        "rrw": smooth((nk + 3, nj + 2 * NG, ni + 2 * NG), 1.5),
    }
    frozen["rrw"][:2] = 0.0
    frozen["rrw"][nk + 1:] = 0.0
    c1 = rng.uniform(0.4, 0.6, (nk + 1, nj, ni)).astype(f32)
    frozen["c1"], frozen["c2"] = c1, (f32(1.0) - c1).astype(f32)
    z = (np.arange(nk) + 0.5) * dz
    shape = (nk, nj, ni)

    def col(x):
        return np.broadcast_to(np.asarray(x, np.float64)[:, None, None], shape).astype(f32).copy()

    rho0 = 1.15 * np.exp(-z / 8500.0)
    frozen["rr0"] = (col(1.0 / rho0) * rng.uniform(0.99, 1.01, shape)).astype(f32)
    frozen["gz"] = rng.uniform(0.98, 1.02, (nj, ni)).astype(f32)
    frozen["divx"] = rng.uniform(-2e-3, 2e-3, shape).astype(f32)
    frozen["th0"] = col(300.0 + 0.004 * z)
    frozen["pi0"] = col(1.0 - 9.81 * z / (cp * 302.0))
    frozen["pp3d"] = rng.uniform(-2e-4, 2e-4, shape).astype(f32)
    pis = frozen["pi0"].astype(np.float64) + frozen["pp3d"]
    prs = p00 * pis ** (cp / rd)
    frozen["prs"] = prs.astype(f32)
    th3d = smooth(shape, 0.8)
    t = (frozen["th0"] + th3d.astype(np.float64)) * pis
    esl = 611.2 * np.exp(17.67 * (t - 273.15) / (t - 29.65))
    qvs = 0.622 * esl / (prs - esl)
    state = {
        "th3d": th3d,
        "qv": (qvs * (1.0 + 0.08 * smooth(shape, 1.0).astype(np.float64))).astype(f32),
        "qc": np.clip(smooth(shape, 1.5e-3, 6e-4), 0.0, None).astype(f32),
        "qr": np.clip(smooth(shape, 2.5e-3, 5e-4), 0.0, None).astype(f32),
    }
    geometry = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, dz=dz, weps=1.0e-6)
    return state, frozen, geometry


def filled_carrier(scalar: np.ndarray, ni: int, nj: int, nk: int) -> np.ndarray:
    """The compact scalar packed into its (nk+2, nj+6, ni+6) carrier with the
    open-side halos filled (west/east columns, then south/north rows)."""
    p = np.zeros((nk + 2, nj + 2 * NG, ni + 2 * NG), np.float32)
    p[1:nk + 1, NG:NG + nj, NG:NG + ni] = scalar
    x0, xl, y0, yl = NG, NG + ni - 1, NG, NG + nj - 1
    for k in range(1, nk + 1):
        for y in range(y0 - 1, yl + 2):
            p[k, y, :x0] = p[k, y, x0]
            p[k, y, xl + 1:] = p[k, y, xl]
        for x in range(x0 - 1, xl + 2):
            p[k, :y0, x] = p[k, y0, x]
            p[k, yl + 1:, x] = p[k, yl, x]
    return p
