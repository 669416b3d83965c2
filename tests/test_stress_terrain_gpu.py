"""The terrain texts' SGS stress and scalar diffusion on the GPU
(gm1_b200/stress.py, csrc/stress_terrain.cu) against the oracle's
restatements (oracle/closure_oracle.c oracle_terrain_strain,
oracle/stress_terrain_oracle.c), which give the reference twins' words on
their goldens: the strain carriers, gettau and turbu/turbv/turbw, and turbs
of theta and the moisture rows, word for word on seeded inputs with
non-flat column metrics (every terrain term live), at 80 levels and on
small ragged grids."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.stress import (launch_cuda_terrain_scalar_turbulence, launch_cuda_terrain_sgs_stress,
                             launch_cuda_terrain_strain, launch_cuda_terrain_stress, terrain_metric_shapes,
                             terrain_scalar_turbulence_workspace, terrain_stress_shapes)
from oracle import stress as ost

pytestmark = pytest.mark.gpu

DX, DY, DZ, DT = 1000.0, 1000.0, 250.0, 5.0


def _metrics(ni, nj, nk, rng):
    f = np.float32
    sh = terrain_metric_shapes(ni, nj, nk)
    m = {}
    for g, r in (("gz", "rgz"), ("gzu", "rgzu"), ("gzv", "rgzv")):
        m[g] = rng.uniform(0.8, 1.25, sh[g]).astype(f)
        m[r] = (f(1.0) / m[g]).astype(f)
    for n in ("gx", "gy", "gxu", "gyv"):
        m[n] = rng.uniform(-0.05, 0.05, sh[n]).astype(f)
    return m


def _stress_inputs(ni, nj, nk, seed):
    rng = np.random.default_rng(seed)
    f = np.float32
    sh = terrain_stress_shapes(ni, nj, nk)
    a = {n: rng.uniform(-3.0, 3.0, sh[n]).astype(f) for n in ("u3d", "v3d", "w3d", "uten", "vten", "wten")}
    a["w3d"] *= f(0.3)
    for n in ("rho", "rf"):
        a[n] = rng.uniform(0.4, 1.2, sh[n]).astype(f)
    for n in ("mh", "mf"):
        a[n] = rng.uniform(0.7, 1.4, sh[n]).astype(f)
    for n in ("kmh", "kmv"):
        a[n] = rng.uniform(1.0, 400.0, sh[n]).astype(f)
    a.update(_metrics(ni, nj, nk, rng))
    for n in ost.STRAIN_NAMES + ost.TAU_NAMES:
        a[n] = np.zeros(sh[n], f)
    return a


def _dev(a):
    return {n: torch.from_numpy(np.ascontiguousarray(v)).cuda() for n, v in a.items()}


def _same(got, want, names):
    bad = {}
    for n in names:
        g = got[n].cpu().numpy()
        if not np.array_equal(g.view(np.uint32), want[n].view(np.uint32)):
            bad[n] = float(np.max(np.abs(g.astype(np.float64) - want[n])))
    assert bad == {}


@pytest.mark.parametrize("ni,nj,nk,seed", [(40, 33, 80, 1), (13, 9, 7, 2), (33, 5, 3, 3), (3, 3, 4, 4)])
def test_terrain_stress_is_the_oracle_word_for_word(ni, nj, nk, seed):
    a = _stress_inputs(ni, nj, nk, seed)
    d = _dev(a)
    ost.terrain_strain(a, ni=ni, nj=nj, nk=nk, dx=DX, dy=DY, dz=DZ)
    launch_cuda_terrain_strain(d, ni=ni, nj=nj, nk=nk, dx=DX, dy=DY, dz=DZ)
    torch.cuda.synchronize()
    # s13/s23 levels 0 and nk are not written by either
    _same(d, a, ("s11", "s22", "s33", "s12"))
    for n in ("s13", "s23"):
        assert np.array_equal(d[n].cpu().numpy()[1:nk].view(np.uint32), a[n][1:nk].view(np.uint32)), n
    ost.terrain_gettau(a, ni=ni, nj=nj, nk=nk)
    ost.terrain_momentum_stress(a, ni=ni, nj=nj, nk=nk, dx=DX, dy=DY, dz=DZ, dt=DT)
    launch_cuda_terrain_stress(d, ni=ni, nj=nj, nk=nk, dx=DX, dy=DY, dz=DZ, dt=DT)
    torch.cuda.synchronize()
    _same(d, a, ost.TAU_NAMES + ("uten", "vten", "wten"))
    assert float(torch.abs(d["uten"] - torch.from_numpy(_stress_inputs(ni, nj, nk, seed)["uten"]).cuda()).max()) > 0


def test_the_chained_terrain_entry_point_is_the_two_passes():
    ni, nj, nk = 21, 17, 12
    a = _stress_inputs(ni, nj, nk, 7)
    d1, d2 = _dev(a), _dev(a)
    launch_cuda_terrain_strain(d1, ni=ni, nj=nj, nk=nk, dx=DX, dy=DY, dz=DZ)
    launch_cuda_terrain_stress(d1, ni=ni, nj=nj, nk=nk, dx=DX, dy=DY, dz=DZ, dt=DT)
    launch_cuda_terrain_sgs_stress(d2, ni=ni, nj=nj, nk=nk, dx=DX, dy=DY, dz=DZ, dt=DT)
    torch.cuda.synchronize()
    for n in ost.TAU_NAMES + ("uten", "vten", "wten", "s11", "s12"):
        assert torch.equal(d1[n].view(torch.int32), d2[n].view(torch.int32)), n


def _turbs_inputs(ni, nj, nk, seed):
    rng = np.random.default_rng(seed)
    f = np.float32
    cell, face = (nk, nj, ni), (nk + 1, nj, ni)
    a = {"th0": np.linspace(300.0, 340.0, nk).astype(f), "tha": rng.uniform(-2.0, 2.0, cell).astype(f),
         "qa": rng.uniform(0.0, 1.4e-2, (6,) + cell).astype(f), "rho": rng.uniform(0.4, 1.2, cell).astype(f),
         "rf": rng.uniform(0.4, 1.2, face).astype(f), "mh": rng.uniform(0.7, 1.4, cell).astype(f),
         "mf": rng.uniform(0.7, 1.4, face).astype(f), "khh": rng.uniform(1.0, 400.0, face).astype(f),
         "khv": rng.uniform(1.0, 400.0, face).astype(f), "thten1": rng.uniform(-1e-3, 1e-3, cell).astype(f),
         "qten": rng.uniform(-1e-6, 1e-6, (6,) + cell).astype(f)}
    a["rr"] = (f(1.0) / a["rho"]).astype(f)
    a.update(_metrics(ni, nj, nk, rng))
    return a


@pytest.mark.parametrize("ni,nj,nk,numq,seed", [(40, 33, 80, 6, 11), (13, 9, 7, 3, 12), (3, 4, 3, 1, 13),
                                                (17, 3, 9, 0, 14)])
def test_terrain_turbs_is_the_oracle_word_for_word(ni, nj, nk, numq, seed):
    a = _turbs_inputs(ni, nj, nk, seed)
    d = _dev(a)
    d["workspace"] = terrain_scalar_turbulence_workspace(ni, nj, nk, numq, d["tha"].device)
    ost.terrain_scalar_turbulence(a, ni=ni, nj=nj, nk=nk, numq=numq, dx=DX, dy=DY, dz=DZ, dt=DT)
    launch_cuda_terrain_scalar_turbulence(d, ni=ni, nj=nj, nk=nk, numq=numq, dx=DX, dy=DY, dz=DZ,
                                          dt=DT)
    torch.cuda.synchronize()
    _same(d, a, ("thten1", "qten"))
    if numq < 6:  # rows past numq untouched
        assert np.array_equal(d["qten"].cpu().numpy()[numq:], _turbs_inputs(ni, nj, nk, seed)["qten"][numq:])


def test_terrain_refusals():
    ni, nj, nk = 8, 7, 6
    d = _dev(_stress_inputs(ni, nj, nk, 5))
    with pytest.raises(ValueError):
        launch_cuda_terrain_stress(d, ni=ni, nj=nj, nk=201, dx=DX, dy=DY, dz=DZ, dt=DT)
    with pytest.raises(ValueError):
        launch_cuda_terrain_stress(d, ni=ni, nj=nj, nk=nk, dx=DX, dy=DY, dz=DZ, dt=0.0)
    bad = dict(d)
    bad["gxu"] = bad["gx"]
    with pytest.raises(Exception):
        launch_cuda_terrain_stress(bad, ni=ni, nj=nj, nk=nk, dx=DX, dy=DY, dz=DZ, dt=DT)
