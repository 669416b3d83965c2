"""The CUDA moist-step pieces through the C ABI against the oracle on
seeded inputs (multi-tile grids): open fills (all six kinds), moist
buoyancy, post-acoustic getdiv/getdivx, the final-stage pdef chain (tile
and open-lateral forms), held composition, solve3 density and scalar pack.
Bar: every float32 word identical, except the held composition's powf
branch (libm vs CUDA powf), compared to 4 float32 ulps of the powf result."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200 import moist_ops as mo
from oracle import moist_step as om
from tests.golden.make_golden import moist_piece_fixture
from tests.test_oracle_moist_step import chain_arrays

pytestmark = pytest.mark.gpu

NI, NJ, NK = 70, 37, 14


def _dev(d):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in d.items()}


def _same(got, want, name):
    g = got.cpu().numpy()
    bad = np.flatnonzero(g.view(np.uint32) != want.view(np.uint32))
    assert bad.size == 0, f"{name}: {bad.size} words differ, first at {np.unravel_index(bad[0], want.shape)}"


@pytest.mark.parametrize("kind", list(om.FILL))
def test_open_fill(kind):
    shapes = {"pressure": (NK + 2, NJ + 2, NI + 2), "scalar": (NK + 2, NJ + 6, NI + 6), "u": (NK + 2, NJ + 6, NI + 7),
              "v": (NK + 2, NJ + 7, NI + 6), "w": (NK + 3, NJ + 6, NI + 6), "w_keep_ends": (NK + 3, NJ + 6, NI + 6)}
    q = np.random.default_rng(3).normal(0, 1, shapes[kind]).astype(np.float32)
    d = torch.from_numpy(q.copy()).cuda()
    om.open_fill(q, kind, ni=NI, nj=NJ, nk=NK)
    mo.open_fill(d, kind, ni=NI, nj=NJ, nk=NK)
    _same(d, q, kind)


def test_moist_buoyancy():
    a = moist_piece_fixture(NI, NJ, NK, 11)
    d = _dev(a)
    names = ("dum8", "c1", "c2", "gxu", "gyv", "uten", "vten", "wten")
    om.moist_buoyancy(*(a[n] for n in names), ni=NI, nj=NJ, nk=NK)
    mo.moist_buoyancy(*(d[n] for n in names), ni=NI, nj=NJ, nk=NK)
    for n in ("uten", "vten", "wten"):
        _same(d[n], a[n], n)


def test_post_acoustic_flux():
    a = moist_piece_fixture(NI, NJ, NK, 12)
    mass = (NK, NJ, NI)
    for n in ("divergence", "theta_divergence_term"):
        a[n] = np.zeros(mass, np.float32)
    d = _dev(a)
    om.post_acoustic_flux(a, ni=NI, nj=NJ, nk=NK, dx=400.0, dy=350.0, dz=180.0)
    mo.post_acoustic_flux(d, ni=NI, nj=NJ, nk=NK, dx=400.0, dy=350.0, dz=180.0)
    for n in ("rru", "rrv", "rrw", "divergence", "theta_divergence_term", "divx"):
        _same(d[n], a[n], n)


@pytest.mark.parametrize("obc,pdefweno", [(0, 1), (0x2222, 0), (0x2222, 1), (0x3141, 1)])
def test_pdef_moisture_chain(obc, pdefweno):
    a = chain_arrays(NI, NJ, NK, 13 + pdefweno)
    d = _dev(a)
    kw = dict(ni=NI, nj=NJ, nk=NK, dttmp=2.0, dx=400.0, dy=300.0, dz=200.0, weps=1e-20, lateral_obc=obc,
              pdefweno=pdefweno)
    om.pdef_moisture_chain(a, **kw)
    mo.pdef_moisture_chain(d, **kw)
    for n in ("fx", "fy", "fz", "advx", "advy", "advz", "candidate", "advection"):
        _same(d[n], a[n], n)


@pytest.mark.parametrize("held_theta", [False, True])
def test_held_compose(held_theta):
    rng = np.random.default_rng(21)
    mass = (NK, NJ, NI)
    a = {"th0": rng.uniform(295, 330, mass), "pi0": rng.uniform(0.7, 1.0, mass), "rho": rng.uniform(0.6, 1.2, mass),
         "ppi": rng.normal(0, 1e-4, mass), "tha": rng.normal(0, 1, mass), "qa": rng.uniform(0, 0.014, (3, *mass)),
         "qpten": rng.normal(0, 1e-7, mass), "qtten": rng.normal(0, 1e-3, mass), "qvten": rng.normal(0, 1e-7, mass),
         "qcten": rng.normal(0, 1e-7, mass), "ppten": np.zeros((NK + 2, NJ + 2, NI + 2)),
         "thheld": rng.normal(0, 1e-3, mass) if held_theta else np.zeros(mass),
         "qheld": np.concatenate([rng.normal(0, 1e-7, (1, *mass)) if held_theta else np.zeros((1, *mass)),
                                  rng.normal(0, 1e-7, (2, *mass))])}
    a = {k: np.ascontiguousarray(v, dtype=np.float32) for k, v in a.items()}
    d = _dev(a)
    om.held_compose(a, ni=NI, nj=NJ, nk=NK, dt=5.0)
    mo.held_compose(d, ni=NI, nj=NJ, nk=NK, dt=5.0)
    _same(d["thheld"], a["thheld"], "thheld")
    _same(d["qheld"], a["qheld"], "qheld")
    if not held_theta:
        _same(d["ppten"], a["ppten"], "ppten")
    else:
        # ppten = (powf(...) - pi0 - ppi) / dt + qpten: the powf result is
        # near 1, so its ulps bound |error| * dt
        got, want = d["ppten"].cpu().numpy().astype(np.float64), a["ppten"].astype(np.float64)
        assert np.max(np.abs(got - want)) * 5.0 <= 4 * 2.0 ** -23


def test_solve3_density_and_pack():
    rng = np.random.default_rng(31)
    rho = rng.uniform(0.6, 1.2, (NK, NJ, NI)).astype(np.float32)
    c1 = rng.uniform(0.4, 0.6, (NK + 1, NJ, NI)).astype(np.float32)
    c2 = (np.float32(1) - c1).astype(np.float32)
    rr, rf = np.zeros_like(rho), np.zeros_like(c1)
    om.solve3_density(rho, c1, c2, rr, rf, ni=NI, nj=NJ, nk=NK)
    d = _dev({"rho": rho, "c1": c1, "c2": c2, "rr": np.zeros_like(rho), "rf": np.zeros_like(c1)})
    mo.solve3_density(d["rho"], d["c1"], d["c2"], d["rr"], d["rf"], ni=NI, nj=NJ, nk=NK)
    _same(d["rr"], rr, "rr")
    _same(d["rf"], rf, "rf")
    s = rng.normal(0, 1, (NK, NJ, NI)).astype(np.float32)
    pad = rng.normal(0, 1, (NK + 2, NJ + 6, NI + 6)).astype(np.float32)
    dp = torch.from_numpy(pad.copy()).cuda()
    om.pack_scalar(s, pad, ni=NI, nj=NJ, nk=NK)
    mo.pack_scalar(torch.from_numpy(s).cuda(), dp, ni=NI, nj=NJ, nk=NK)
    _same(dp, pad, "padded")


@pytest.mark.parametrize("flat", [False, True])
@pytest.mark.parametrize("obc", [0x2222, 0])
def test_pdef_moisture_chain_on_a_stretched_column(flat, obc):
    """The chain with the terrain branch's rdsf(k) or the flat column's
    rdz*mh(k) (seeded profiles) against the oracle restatement, word for word."""
    from gm1_b200.advection import StretchedColumn

    a = chain_arrays(NI, NJ, NK, 17)
    d = _dev(a)
    rng = np.random.default_rng(19)
    rdsf = np.zeros(NK + 3, np.float32)
    rdsf[1:NK + 1] = rng.uniform(1.0 / 600.0, 1.0 / 40.0, NK).astype(np.float32)
    mh = rng.uniform(0.3, 3.0, NK + 2).astype(np.float32)
    rdz = float(np.float32(1.0) / np.float32(100.0))
    kw = dict(ni=NI, nj=NJ, nk=NK, dttmp=2.0, dx=400.0, dy=300.0, weps=1e-20, lateral_obc=obc, pdefweno=1)
    om.pdef_moisture_chain_column(a, flat=flat, profile=mh if flat else rdsf, rdz=rdz, **kw)
    column = (StretchedColumn(flat=True, mh=torch.from_numpy(mh).cuda(), rdz=rdz) if flat
              else StretchedColumn(flat=False, rdsf=torch.from_numpy(rdsf).cuda()))
    mo.pdef_moisture_chain_column(d, column, **kw)
    for n in ("fx", "fy", "fz", "advx", "advy", "advz", "candidate", "advection"):
        _same(d[n], a[n], n)


@pytest.mark.parametrize("flat", [False, True])
def test_post_acoustic_flux_on_a_stretched_column(flat):
    """getdiv/getdivx on a generated stretched column (terrain branch or flat)
    against the oracle restatement of the reference's stretched texts, word
    for word; and the flat column's w-only buoyancy."""
    from gm1_b200.momentum import StretchedMomentumColumn
    from gm1_b200.vertical import build_vertical_levels
    from tests.test_oracle_momentum import _padded_rho0

    a = moist_piece_fixture(NI, NJ, NK, 31)
    mass = (NK, NJ, NI)
    for n in ("divergence", "theta_divergence_term"):
        a[n] = np.zeros(mass, np.float32)
    lv = build_vertical_levels(stretch_z=1, nk=NK, dz_m=100.0, ztop_m=1630.0, str_bot_m=40.0, str_top_m=1030.0,
                               dz_bot_m=20.0, dz_top_m=200.0)
    rho0p = _padded_rho0(a["rho0_3d"], NI, NJ, NK)
    rdz = float(np.float32(1.0) / np.float32(100.0))
    col = {"flat": flat, "rho0p": rho0p, "sigma": lv.sigma, "sigmaf": lv.sigmaf, "rds": lv.rds, "rdsf": lv.rdsf,
           "ztop": lv.ztop_m, "mh": lv.mh, "rdz": rdz}
    d = _dev(a)
    om.post_acoustic_flux_column(a, col, ni=NI, nj=NJ, nk=NK, dx=400.0, dy=350.0)
    t = lambda x: torch.from_numpy(np.array(x, dtype=np.float32)).cuda()  # noqa: E731
    vertical = (StretchedMomentumColumn(True, t(rho0p), mh=t(lv.mh), rdz=rdz) if flat else
                StretchedMomentumColumn(False, t(rho0p), sigma=t(lv.sigma), sigmaf=t(lv.sigmaf), rds=t(lv.rds),
                                        rdsf=t(lv.rdsf), ztop=lv.ztop_m))
    mo.post_acoustic_flux_column(d, vertical, ni=NI, nj=NJ, nk=NK, dx=400.0, dy=350.0)
    for n in ("rru", "rrv", "rrw", "divergence", "theta_divergence_term", "divx"):
        _same(d[n], a[n], n)
    if flat:
        b = moist_piece_fixture(NI, NJ, NK, 11)
        db = _dev(b)
        om.moist_buoyancy_flat(b["dum8"], b["c1"], b["c2"], b["wten"], ni=NI, nj=NJ, nk=NK)
        mo.moist_buoyancy_flat(db["dum8"], db["c1"], db["c2"], db["wten"], ni=NI, nj=NJ, nk=NK)
        _same(db["wten"], b["wten"], "wten")
