"""Parity of the CUDA closure inputs (calcdef, calcnm) through the C ABI with
the reference's CPU twins (golden fixtures) and with the oracle on larger,
multi-tile grids.  Bars as in tests/test_oracle_closure.py: calcdef word for
word; calcnm cell outputs, saturation mask and branch counts word for word,
nm within NM_MAX_REL of max|nm| (device logf/expf)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.closure import launch_cuda_moist_nm, launch_cuda_terrain_deformation
from oracle import closure as orc
from tests.golden.make_golden import deformation_fixture, moist_nm_fixture
from tests.test_oracle_closure import NM_EXACT, NM_MAX_REL, load, nm_error

pytestmark = pytest.mark.gpu


def _dev(a):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in a.items()}


def _run_calcdef(a, meta):
    dev = _dev(a)
    launch_cuda_terrain_deformation(dev, **{k: meta[k] for k in ("ni", "nj", "nk", "dx", "dy", "dz")})
    torch.cuda.synchronize()
    return {n: dev[n].cpu().numpy() for n in ("defv", "defh")}


def _run_nm(a, meta):
    dev = _dev(a)
    counts = torch.zeros(4, dtype=torch.int64, device="cuda")
    launch_cuda_moist_nm(dev, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dz=meta["dz"], counts=counts)
    torch.cuda.synchronize()
    got = {n: dev[n].cpu().numpy() for n in ("nm",) + NM_EXACT + ("saturation_mask",)}
    return got, [int(x) for x in counts.cpu()]


@pytest.mark.parametrize("tag", ["calcdef_9x7x8", "calcdef_12x6x10"])
def test_calcdef_bit_exact_vs_reference(tag):
    meta, a, want = load(tag)
    got = _run_calcdef(a, meta)
    for n in ("defv", "defh"):
        assert np.array_equal(got[n].view(np.uint32), want[n].view(np.uint32)), n


@pytest.mark.parametrize("shape", [(70, 45, 12), (33, 9, 3), (5, 4, 3)])
def test_calcdef_bit_exact_vs_oracle_multi_tile(shape):
    ni, nj, nk = shape
    a = deformation_fixture(ni, nj, nk, seed=ni + nj + nk)
    dx, dy, dz = (float(x) for x in a.pop("_spacing"))
    meta = {"ni": ni, "nj": nj, "nk": nk, "dx": dx, "dy": dy, "dz": dz}
    got = _run_calcdef(a, meta)
    orc.calcdef(a, **meta)
    for n in ("defv", "defh"):
        assert np.array_equal(got[n].view(np.uint32), a[n].view(np.uint32)), n


@pytest.mark.parametrize("tag", ["moist_nm_8x6x14", "moist_nm_5x9x20"])
def test_moist_nm_vs_reference(tag):
    meta, a, want = load(tag)
    got, counts = _run_nm(a, meta)
    assert counts == [meta[k] for k in ("saturated", "liquid", "mixed", "ice")]
    for n in NM_EXACT:
        assert np.array_equal(got[n].view(np.uint32), want[n].view(np.uint32)), n
    assert np.array_equal(got["saturation_mask"], want["saturation_mask"])
    assert nm_error(got["nm"], want["nm"]) <= NM_MAX_REL


def test_moist_nm_vs_oracle_large():
    ni, nj, nk = 67, 33, 30
    a = moist_nm_fixture(ni, nj, nk, seed=61)
    got, counts = _run_nm(a, {"ni": ni, "nj": nj, "nk": nk, "dz": 200.0})
    ref = orc.moist_nm(a, ni=ni, nj=nj, nk=nk, dz=200.0)
    assert counts == [ref[k] for k in ("saturated", "liquid", "mixed", "ice")]
    for n in NM_EXACT:
        assert np.array_equal(got[n].view(np.uint32), a[n].view(np.uint32)), n
    assert np.array_equal(got["saturation_mask"], a["saturation_mask"])
    assert nm_error(got["nm"], a["nm"]) <= NM_MAX_REL
    assert not np.any(got["nm"][0]) and not np.any(got["nm"][nk])
