"""Pins of the moist-step pieces of the oracle: the open-lateral fills
against the reference's own cpu_bc*_open_inplace (golden), and the interior
of the final-stage pdef chain against the twin-pinned pdef direction
(cpu_pdef_direction_inplace restated in rk_oracle.c): fed the chain's own
directional advection, it must leave the same words the chain leaves on
every interior cell of every axis.  The chain's fluxes, the moist buoyancy
and getdiv/getdivx restate the reference's kernel source (no CPU twin
exists for them)."""

from __future__ import annotations

import json

import numpy as np
import pytest

from oracle import moist_step as om
from oracle import rk as rk
from tests._golden import GOLDEN
from tests.golden.make_golden import moist_piece_fixture


@pytest.mark.parametrize("kind", list(om.FILL))
def test_fill_matches_reference(kind):
    z = np.load(GOLDEN / "open_fills_9x7x6.npz")
    meta = json.loads(str(z["meta"]))
    q = z[f"in_{kind}"].copy()
    om.open_fill(q, kind, **meta)
    assert np.array_equal(q.view(np.uint32), z[f"out_{kind}"].view(np.uint32))


def chain_arrays(ni, nj, nk, seed):
    a = moist_piece_fixture(ni, nj, nk, seed)
    mass, su, sv, sw = (nk, nj, ni), a["rru"].shape, a["rrv"].shape, a["rrw"].shape
    c = {n: a[n] for n in ("scalar_a", "scalar_padded", "rho0_3d", "gz", "rgz", "rr0", "c1", "c2", "divx", "rru",
                           "rrv", "rrw")}
    c.update(fx=np.zeros(su, np.float32), fy=np.zeros(sv, np.float32), fz=np.zeros(sw, np.float32),
             advx=np.zeros(mass, np.float32), advy=np.zeros(mass, np.float32), advz=np.zeros(mass, np.float32),
             candidate=np.zeros(mass, np.float32), advection=np.zeros(mass, np.float32))
    return c


def test_chain_interior_matches_twin_pinned_pdef_direction():
    ni, nj, nk = 13, 11, 10
    kw = dict(ni=ni, nj=nj, nk=nk, dttmp=2.0, dx=400.0, dy=300.0, dz=200.0, weps=1e-20, lateral_obc=0, pdefweno=1)
    pre = chain_arrays(ni, nj, nk, 5)
    om.pdef_moisture_directional(pre, **kw)
    full = chain_arrays(ni, nj, nk, 5)
    om.pdef_moisture_chain(full, **kw)
    flux = {"x": pre["rru"], "y": pre["rrv"], "z": pre["rrw"]}
    spacing = {"x": 400.0, "y": 300.0, "z": 200.0}
    repaired = 0
    for axis, name in (("x", "advx"), ("y", "advy"), ("z", "advz")):
        d = pre[name].copy()
        cand = np.zeros_like(d)
        rk.pdef_direction(pre["scalar_a"], pre["scalar_padded"], pre["rho0_3d"], pre["gz"], pre["rgz"], flux[axis], d,
                          cand, axis=axis, dt=2.0, spacing=spacing[axis])
        inner = (slice(None), slice(1, nj - 1), slice(1, ni - 1)) if axis != "z" else (slice(None),) * 3
        assert np.array_equal(d[inner].view(np.uint32), full[name][inner].view(np.uint32)), axis
        repaired += int(np.count_nonzero(d != pre[name]))
    assert repaired > 0


def test_chain_with_open_sides_fills_every_cell():
    ni, nj, nk = 12, 9, 8
    a = chain_arrays(ni, nj, nk, 6)
    a["advection"][:] = np.nan
    om.pdef_moisture_chain(a, ni=ni, nj=nj, nk=nk, dttmp=1.5, dx=250.0, dy=250.0, dz=150.0, weps=1e-20,
                           lateral_obc=0x2222, pdefweno=0)
    assert np.isfinite(a["advection"]).all()


@pytest.mark.parametrize("obc", [0x2222, 0])
def test_chain_on_uniform_columns_is_the_uniform_chain(obc):
    """The stretched-column chain (restatement of the reference's
    profile-bound pdef texts) reduces word for word to the uniform chain: a
    terrain column whose rdsf(k) is 1/dz, and a flat column (mh = 1,
    rdz = 1/dz) over a horizontally uniform base state with flat metrics."""
    ni, nj, nk = 12, 10, 9
    dz = 200.0
    kw = dict(ni=ni, nj=nj, nk=nk, dttmp=2.0, dx=400.0, dy=300.0, weps=1e-20, lateral_obc=obc, pdefweno=1)
    rdz = float(np.float32(1.0) / np.float32(dz))
    for flat in (False, True):
        a = chain_arrays(ni, nj, nk, 23)
        if flat:
            a["rho0_3d"][:] = a["rho0_3d"][:, :1, :1]
            a["rr0"][:] = a["rr0"][:, :1, :1]
            a["gz"][:] = np.float32(1.0)
            a["rgz"][:] = np.float32(1.0)
        want = {k: v.copy() for k, v in a.items()}
        om.pdef_moisture_chain(want, dz=dz, **kw)
        prof = np.ones(nk + 2, np.float32) if flat else np.full(nk + 3, np.float32(rdz), np.float32)
        om.pdef_moisture_chain_column(a, flat=flat, profile=prof, rdz=rdz, **kw)
        for n in ("advx", "advy", "advz", "candidate", "advection"):
            assert np.array_equal(a[n].view(np.uint32), want[n].view(np.uint32)), (flat, n)


def test_post_acoustic_on_the_uniform_terrain_column_is_the_uniform_operator():
    """The stretched getdiv/getdivx restatement on the uniform column's own
    profile words and a clamped-halo padded density reduces word for word to
    the uniform post-acoustic flux."""
    from gm1_b200.vertical import uniform_vertical_levels
    from tests.test_oracle_momentum import _padded_rho0

    ni, nj, nk, dz = 14, 11, 9, 180.0
    a = moist_piece_fixture(ni, nj, nk, 12)
    for n in ("divergence", "theta_divergence_term"):
        a[n] = np.zeros((nk, nj, ni), np.float32)
    b = {k: v.copy() for k, v in a.items()}
    om.post_acoustic_flux(a, ni=ni, nj=nj, nk=nk, dx=400.0, dy=350.0, dz=dz)
    lv = uniform_vertical_levels(nk, dz)
    col = {"flat": False, "rho0p": _padded_rho0(b["rho0_3d"], ni, nj, nk), "sigma": lv.sigma, "sigmaf": lv.sigmaf,
           "rds": lv.rds, "rdsf": lv.rdsf, "ztop": lv.ztop_m}
    om.post_acoustic_flux_column(b, col, ni=ni, nj=nj, nk=nk, dx=400.0, dy=350.0)
    for n in ("rru", "rrv", "rrw", "divergence", "theta_divergence_term", "divx"):
        assert np.array_equal(a[n].view(np.uint32), b[n].view(np.uint32)), n


def test_oracle_initial_state_is_the_package_state_word_for_word():
    """The benchmark's CPU baseline and reference arm build their inputs with
    oracle.moist_initial (no CUDA library on that path); it must give the
    package's starting state and metrics word for word (the package's
    column is host code in the library, so this runs without a GPU)."""
    from gm1_b200.moist_step import MoistStepConfig, weisman_klemp_initial_state
    from oracle.moist_initial import weisman_klemp_initial_state as oracle_state

    cfg = MoistStepConfig(20, 14, 12, 1000.0, 1000.0, 250.0, 5.0, 10)
    kw = dict(seed=2, bubble_k=3.0, noise_k=0.1, bubble_radius_m=(6000.0, 1500.0), bubble_center_z_m=1500.0,
              bubble_cloud=1.0e-3, bubble_rain=5.0e-4)
    hs, hm = weisman_klemp_initial_state(cfg, **kw)
    os_, om_ = oracle_state(cfg, **kw)
    assert sorted(hs) == sorted(os_) and sorted(hm) == sorted(om_)
    for n in hs:
        assert hs[n].dtype == os_[n].dtype and hs[n].shape == os_[n].shape, n
        assert np.array_equal(hs[n].view(np.uint8), os_[n].view(np.uint8)), n
    for n in hm:
        assert np.array_equal(hm[n].view(np.uint8), om_[n].view(np.uint8)), n


def test_oracle_stretched_initial_state_is_the_package_state_word_for_word():
    """The same on a stretched column (stretch_z 1, 20 m at the ground):
    the state, the metrics, the column profiles and the padded base density."""
    from gm1_b200.moist_step import MoistStepConfig, StretchedColumnSpec, weisman_klemp_initial_state
    from oracle.moist_initial import weisman_klemp_initial_state as oracle_state

    cfg = MoistStepConfig(18, 12, 14, 100.0, 100.0, 100.0, 0.6, 8,
                          column=StretchedColumnSpec(1630.0, 40.0, 1030.0, 20.0, 200.0))
    kw = dict(seed=3, bubble_radius_m=(600.0, 500.0), bubble_center_z_m=500.0, bubble_cloud=1.0e-3)
    hs, hm = weisman_klemp_initial_state(cfg, **kw)
    os_, om_ = oracle_state(cfg, **kw)
    assert sorted(hs) == sorted(os_) and sorted(hm) == sorted(om_)
    for d1, d2 in ((hs, os_), (hm, om_)):
        for n in d1:
            assert d1[n].shape == d2[n].shape, n
            assert np.array_equal(d1[n].view(np.uint8), d2[n].view(np.uint8)), n
    assert float(hm["mh"].max()) > float(hm["mh"].min())  # stretched
