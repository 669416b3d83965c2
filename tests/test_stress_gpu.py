"""The flat-column SGS stress on the GPU (gm1_b200/stress.py, csrc/stress.cu)
against the oracle's restatement (oracle/stress_oracle.c): the strain
carriers, gettau and turbu/turbv/turbw word for word on seeded inputs with
the stretched 20-500 m column's metrics, at 80 levels and on small ragged
grids; the argument refusals."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.errors import CM1Refusal
from gm1_b200.stress import (launch_cuda_flat_gettau, launch_cuda_flat_momentum_stress, launch_cuda_flat_sgs_stress,
                             launch_cuda_flat_strain)
from oracle import stress as ost

pytestmark = pytest.mark.gpu

DX, DT = 100.0, 0.6


def _column(nk):
    """mh/mf profiles of the 20-500 m stretched column (or a made-up
    stretching when nk is small) and the coordinate's rdz."""
    if nk == 80:
        from gm1_b200.vertical import build_vertical_levels

        lv = build_vertical_levels(stretch_z=1, nk=80, dz_m=100.0, ztop_m=20800.0, str_bot_m=200.0,
                                   str_top_m=15800.0, dz_bot_m=20.0, dz_top_m=500.0)
        return np.asarray(lv.mh[1:nk + 1], np.float32), np.asarray(lv.mf[1:nk + 2], np.float32), 0.01
    z = np.linspace(0.0, 1.0, nk + 1)
    mf = (1.0 / (0.3 + 1.4 * z)).astype(np.float32)
    mh = (0.5 * (mf[:-1] + mf[1:])).astype(np.float32)
    return mh, mf, 0.002


def _inputs(ni, nj, nk, seed):
    rng = np.random.default_rng(seed)
    sh = ost.stress_shapes(ni, nj, nk)
    f = np.float32
    mh, mf, rdz = _column(nk)
    a = {n: np.zeros(sh[n], f) for n in sh}
    a["u3d"][:] = rng.normal(5.0, 3.0, sh["u3d"])
    a["v3d"][:] = rng.normal(-2.0, 3.0, sh["v3d"])
    a["w3d"][1:nk] = rng.normal(0.0, 1.0, (nk - 1, nj, ni))
    a["rho"][:] = np.linspace(1.15, 0.2, nk, dtype=f)[:, None, None] * rng.uniform(0.98, 1.02, sh["rho"])
    a["rf"][:] = np.linspace(1.16, 0.19, nk + 1, dtype=f)[:, None, None] * rng.uniform(0.98, 1.02, sh["rf"])
    a["mh"][:] = mh[:, None, None]
    a["mf"][:] = mf[:, None, None]
    a["mh_profile"][1:nk + 1] = mh
    a["mh_profile"][0], a["mh_profile"][nk + 1] = mh[0], mh[-1]
    a["kmh"][:] = rng.uniform(0.0, 60.0, sh["kmh"])
    a["kmv"][:] = rng.uniform(0.0, 60.0, sh["kmv"])
    for n in ost.TENDENCY_NAMES:
        a[n][:] = rng.normal(0.0, 1e-3, sh[n])
    return a, rdz


def _dev(a):
    return {n: torch.from_numpy(v.copy()).cuda() for n, v in a.items()}


def _same(got, want, names):
    bad = {}
    for n in names:
        g = got[n].cpu().numpy()
        if not np.array_equal(g.view(np.uint32), want[n].view(np.uint32)):
            bad[n] = int(np.count_nonzero(g.view(np.uint32) != want[n].view(np.uint32)))
    assert not bad, bad


@pytest.mark.parametrize("ni,nj,nk,seed", [(64, 48, 80, 1), (13, 9, 7, 2), (33, 5, 3, 3), (3, 3, 4, 4)])
def test_each_pass_is_the_oracle_word_for_word(ni, nj, nk, seed):
    a, rdz = _inputs(ni, nj, nk, seed)
    d = _dev(a)
    ost.flat_strain(a, ni=ni, nj=nj, nk=nk, dx=DX, dy=DX, rdz=rdz)
    launch_cuda_flat_strain(d, ni=ni, nj=nj, nk=nk, dx=DX, dy=DX, rdz=rdz)
    torch.cuda.synchronize()
    _same(d, a, ost.STRAIN_NAMES)
    ost.flat_gettau(a, ni=ni, nj=nj, nk=nk)
    launch_cuda_flat_gettau(d, ni=ni, nj=nj, nk=nk)
    torch.cuda.synchronize()
    _same(d, a, ost.TAU_NAMES)
    ost.flat_momentum_stress(a, ni=ni, nj=nj, nk=nk, dx=DX, dy=DX, rdz=rdz, dt=DT)
    launch_cuda_flat_momentum_stress(d, ni=ni, nj=nj, nk=nk, dx=DX, dy=DX, rdz=rdz, dt=DT)
    torch.cuda.synchronize()
    _same(d, a, ost.TENDENCY_NAMES)
    assert np.any(a["uten"] != _inputs(ni, nj, nk, seed)[0]["uten"])


def test_the_chained_entry_point_is_the_three_passes():
    ni, nj, nk = 40, 36, 80
    a, rdz = _inputs(ni, nj, nk, 7)
    d = _dev(a)
    ost.flat_sgs_stress(a, ni=ni, nj=nj, nk=nk, dx=DX, dy=DX, rdz=rdz, dt=DT)
    launch_cuda_flat_sgs_stress(d, ni=ni, nj=nj, nk=nk, dx=DX, dy=DX, rdz=rdz, dt=DT)
    torch.cuda.synchronize()
    _same(d, a, ost.STRAIN_NAMES + ost.TAU_NAMES + ost.TENDENCY_NAMES)


def test_refusals():
    ni, nj, nk = 8, 8, 6
    a, rdz = _inputs(ni, nj, nk, 8)
    d = _dev(a)
    with pytest.raises(CM1Refusal):
        launch_cuda_flat_momentum_stress(d, ni=ni, nj=nj, nk=nk, dx=DX, dy=DX, rdz=rdz, dt=DT, two_part=object())
    with pytest.raises(ValueError):
        launch_cuda_flat_momentum_stress(d, ni=ni, nj=nj, nk=nk, dx=DX, dy=DX, rdz=rdz, dt=-1.0)
    bad = dict(d)
    bad["t12"] = d["t12"][:, :-1]
    with pytest.raises(ValueError):
        launch_cuda_flat_gettau(bad, ni=ni, nj=nj, nk=nk)
    with pytest.raises(ValueError):
        launch_cuda_flat_momentum_stress({**d, "vten": d["uten"]}, ni=ni, nj=nj, nk=nk, dx=DX, dy=DX, rdz=rdz, dt=DT)


# ------------------------------------------------------------------ turbs
def _turbs_inputs(ni, nj, nk, numq, seed):
    rng = np.random.default_rng(seed)
    f = np.float32
    mh, mf, rdz = _column(nk)
    mass, face = (nk, nj, ni), (nk + 1, nj, ni)
    a = {"th0": np.linspace(300.0, 345.0, nk).astype(f), "tha": rng.normal(0.0, 2.0, mass).astype(f),
         "qa": np.abs(rng.normal(0.0, 5e-3, (6, nk, nj, ni))).astype(f),
         "rho": (np.linspace(1.15, 0.2, nk, dtype=f)[:, None, None] * rng.uniform(0.98, 1.02, mass)).astype(f),
         "rf": (np.linspace(1.16, 0.19, nk + 1, dtype=f)[:, None, None] * rng.uniform(0.98, 1.02, face)).astype(f),
         "mh": np.broadcast_to(mh[:, None, None], mass).astype(f), "mf": np.broadcast_to(mf[:, None, None], face).astype(f),
         "khh": rng.uniform(0.0, 90.0, face).astype(f), "khv": rng.uniform(0.0, 90.0, face).astype(f),
         "thten1": rng.normal(0.0, 1e-3, mass).astype(f), "qten": rng.normal(0.0, 1e-7, (numq, nk, nj, ni)).astype(f)}
    a["rr"] = (f(1.0) / a["rho"]).astype(f)
    return a, float(np.float32(1.0) / np.float32(rdz))


@pytest.mark.parametrize("ni,nj,nk,numq,seed", [(64, 48, 80, 3, 11), (13, 9, 7, 6, 12), (3, 4, 3, 1, 13),
                                                (17, 3, 5, 0, 14)])
def test_flat_turbs_is_the_oracle_word_for_word(ni, nj, nk, numq, seed):
    from gm1_b200.stress import launch_cuda_flat_scalar_turbulence

    from gm1_b200.stress import scalar_turbulence_workspace

    a, dz = _turbs_inputs(ni, nj, nk, numq, seed)
    d = _dev(a)
    d["workspace"] = scalar_turbulence_workspace(ni, nj, nk, numq, d["tha"].device)
    ost.flat_scalar_turbulence(a, ni=ni, nj=nj, nk=nk, numq=numq, dx=DX, dy=DX, dz=dz, dt=DT)
    launch_cuda_flat_scalar_turbulence(d, ni=ni, nj=nj, nk=nk, numq=numq, dx=DX, dy=DX, dz=dz, dt=DT)
    torch.cuda.synchronize()
    _same(d, a, ("thten1", "qten"))
    assert np.array_equal(d["qa"].cpu().numpy(), a["qa"])


# --------------------------------------------------------------- Rayleigh
@pytest.mark.parametrize("profiles,add_momentum", [(False, False), (True, False), (True, True)])
def test_rayleigh_held_is_the_oracle_word_for_word(profiles, add_momentum):
    from gm1_b200.rayleigh import build_rayleigh_coefficients, launch_cuda_rayleigh_held

    ni, nj, nk = 70, 33, 80
    rng = np.random.default_rng(21)
    f = np.float32
    zf = np.concatenate([[0.0], np.cumsum(np.linspace(20.0, 500.0, nk))]).astype(f)
    zh = (0.5 * (zf[:-1] + zf[1:])).astype(f)
    tauh, taus, tauf = build_rayleigh_coefficients(zh, zf, damping_start_m=15000.0)
    if not profiles:
        tauh, taus, tauf = (np.ascontiguousarray(np.broadcast_to(t[:, None, None], (t.shape[0], nj + 2, ni + 2)))
                            for t in (tauh, taus, tauf))
    a = {"tauh": tauh, "taus": taus, "tauf": tauf, "u0": rng.normal(5, 8, nk).astype(f),
         "v0": rng.normal(0, 4, nk).astype(f), "ua": rng.normal(6, 9, (nk, nj, ni + 1)).astype(f),
         "va": rng.normal(0, 5, (nk, nj + 1, ni)).astype(f), "wa": rng.normal(0, 2, (nk, nj, ni)).astype(f),
         "tha": rng.normal(0, 2, (nk, nj, ni)).astype(f), "uten1": rng.normal(0, 1e-3, (nk, nj, ni + 1)).astype(f),
         "vten1": rng.normal(0, 1e-3, (nk, nj + 1, ni)).astype(f), "wten1": rng.normal(0, 1e-3, (nk, nj, ni)).astype(f),
         "thten1": rng.normal(0, 1e-3, (nk, nj, ni)).astype(f)}
    d = _dev(a)
    ost.rayleigh_held(a, ni=ni, nj=nj, nk=nk, rdalpha=1.0 / 300.0, profiles=profiles, add_momentum=add_momentum)
    launch_cuda_rayleigh_held(d, ni=ni, nj=nj, nk=nk, rdalpha=1.0 / 300.0, profiles=profiles,
                              add_momentum=add_momentum)
    torch.cuda.synchronize()
    _same(d, a, ("uten1", "vten1", "wten1", "thten1"))
    assert np.count_nonzero(a["thten1"]) > 0


# ---------------------------------------------------- dissipative heating
def test_dissipative_heating_is_the_oracle_word_for_word():
    from gm1_b200.stress import launch_cuda_dissipative_heating

    ni, nj, nk = 70, 33, 80
    rng = np.random.default_rng(31)
    f = np.float32
    a = {"dissten": rng.uniform(0.0, 0.05, (nk + 1, nj, ni)).astype(f), "pi0": np.linspace(1.0, 0.4, nk).astype(f),
         "ppi": rng.normal(0.0, 2e-3, (nk, nj, ni)).astype(f), "qa": np.abs(rng.normal(0, 3e-3, (6, nk, nj, ni))).astype(f),
         "thten1": rng.normal(0.0, 1e-3, (nk, nj, ni)).astype(f)}
    d = _dev(a)
    ost.dissipative_heating(a, ni=ni, nj=nj, nk=nk)
    launch_cuda_dissipative_heating(d, ni=ni, nj=nj, nk=nk)
    torch.cuda.synchronize()
    _same(d, a, ("thten1",))
