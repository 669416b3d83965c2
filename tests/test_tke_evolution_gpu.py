"""Parity of the CUDA TKE evolution (turbt, RK stages, commit) through the C
ABI with the reference's CPU twin (golden fixtures: tketen, per-stage
digests, committed fields) and with the oracle on a larger multi-tile grid.
Bar: every float32 word identical."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest
import torch

from gm1_b200 import tke_evolution as te
from oracle import tke_evolution as orc
from tests.golden.make_golden import tke_evolution_fixture
from tests.test_oracle_tke_evolution import PARAMS, load

pytestmark = pytest.mark.gpu


def _dev(a):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in a.items()}


def _digest(t):
    return hashlib.sha256(t.cpu().numpy().astype("<f4", copy=False).tobytes()).hexdigest()


@pytest.mark.parametrize("tag", ["tke_evolution_9x8x10", "tke_evolution_7x10x9"])
def test_frozen_flux_operator_bit_exact_vs_reference(tag):
    meta, a, want = load(tag)
    dev = _dev(a)
    te.launch_cuda_tke_evolution_frozen_flux(dev, **{k: meta[k] for k in PARAMS})
    torch.cuda.synchronize()
    for n in ("tketen", "tke3d", "tkea"):
        got = dev[n].cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want[n].view(np.uint32)), n


@pytest.mark.parametrize("tag", ["tke_evolution_9x8x10", "tke_evolution_7x10x9"])
def test_stage_by_stage_matches_reference_stage_digests(tag):
    meta, a, want = load(tag)
    dev = _dev(a)
    p = {k: meta[k] for k in PARAMS}
    ws = torch.empty_like(dev["tke3d"])
    te.launch_cuda_tke_diffusion(dev, **p)
    digests = []
    for nrk in (1, 2, 3):
        te.launch_cuda_tke_rk_stage(dev, workspace=ws, nrk=nrk, **p)
        torch.cuda.synchronize()
        digests.append(_digest(dev["tke3d"]))
    te.launch_cuda_tke_commit(dev, ni=p["ni"], nj=p["nj"], nk=p["nk"], completed_nrk=3)
    torch.cuda.synchronize()
    assert digests == meta["stage_sha256"]
    assert np.array_equal(dev["tkea"].cpu().numpy().view(np.uint32), want["tkea"].view(np.uint32))


def test_operator_bit_exact_vs_oracle_multi_tile():
    ni, nj, nk = 70, 37, 20
    a = tke_evolution_fixture(ni, nj, nk, seed=79)
    p = {"ni": ni, "nj": nj, "nk": nk, "dx": 500.0, "dy": 450.0, "dz": 150.0, "dt": 2.0}
    dev = _dev(a)
    te.launch_cuda_tke_evolution_frozen_flux(dev, **p)
    orc.tke_evolution(a, **p)
    torch.cuda.synchronize()
    for n in ("tketen", "tke3d", "tkea"):
        assert np.array_equal(dev[n].cpu().numpy().view(np.uint32), a[n].view(np.uint32)), n
