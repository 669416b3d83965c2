"""Parity of the CUDA terrain/open momentum advection through the C ABI with
the reference's CPU twin (golden fixtures, three lateral families) and with
the oracle on larger multi-tile grids, the minimum grid, and the split
(hooked) entry.  Bar: every float32 word identical."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200 import momentum as mom
from oracle import momentum as orc
from tests.golden.make_golden import momentum_fixture
from tests.test_oracle_momentum import OUTS, TAGS, load

pytestmark = pytest.mark.gpu


def _dev(a):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in a.items()}


def _same(got, want, name):
    g = got.cpu().numpy() if isinstance(got, torch.Tensor) else got
    bad = np.flatnonzero(g.view(np.uint32) != want.view(np.uint32))
    assert bad.size == 0, f"{name}: {bad.size} words differ, first at {np.unravel_index(bad[0], want.shape)}"


@pytest.mark.parametrize("tag", TAGS)
def test_operator_bit_exact_vs_reference(tag):
    meta, a, want = load(tag)
    dev = _dev(a)
    out = mom.launch_cuda_terrain_open_momentum_advection5(
        dev, dev, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], nrk=1, dx=meta["dx"], dy=meta["dy"], dz=meta["dz"],
        lateral_sides=tuple(meta["lateral_sides"]))
    out.ready_event.synchronize()
    for n in OUTS:
        _same(out.divx if n == "divx" else dev[n], want[n], n)


@pytest.mark.parametrize("ni,nj,nk,sides", [(70, 40, 20, (2, 2, 2, 2)), (70, 40, 20, (1, 1, 1, 1)),
                                            (67, 45, 17, (3, 4, 2, 3)), (7, 7, 8, (2, 3, 4, 2)),
                                            (7, 7, 8, (1, 1, 1, 1))])
def test_operator_bit_exact_vs_oracle(ni, nj, nk, sides):
    a, m, _ = momentum_fixture(ni, nj, nk, 1000 + ni + nk)
    dev = _dev({**a, **m})
    divx = torch.full((nk, nj, ni), float("nan"), device="cuda")
    mom.launch_cuda_terrain_open_momentum_advection5(dev, dev, ni=ni, nj=nj, nk=nk, nrk=2, dx=500.0, dy=450.0,
                                                     dz=150.0, divx=divx, lateral_sides=sides)
    ref = {**a, **m, "divx": np.zeros((nk, nj, ni), np.float32)}
    orc.momentum_advection5(ref, ni=ni, nj=nj, nk=nk, dx=500.0, dy=450.0, dz=150.0, lateral_sides=sides)
    torch.cuda.synchronize()
    for n in OUTS:
        _same(divx if n == "divx" else dev[n], ref[n], n)


def test_hooked_split_entry_matches_one_call():
    ni, nj, nk, sides = 40, 33, 12, (2, 2, 1, 1)
    a, m, _ = momentum_fixture(ni, nj, nk, 7)
    one, two = _dev({**a, **m}), _dev({**a, **m})
    kw = dict(ni=ni, nj=nj, nk=nk, nrk=3, dx=400.0, dy=400.0, dz=200.0, lateral_sides=sides)
    r1 = mom.launch_cuda_terrain_open_momentum_advection5(one, one, **kw)
    seen = []

    def rrw_hook(rrw, *, stream, ni, nj, nk):
        seen.append("rrw")
        return {"performed": True, "flag": 0, "vertical_rigid_faces_written": False,
                "stream_pointer": int(stream.cuda_stream), "schema": "gm1.cuda-bcw-rrw-open-flag0/v1",
                "directions": ["west", "east", "south", "north"]}

    def post_hook(arrays, *, stream, ni, nj, nk, nrk, ng):
        seen.append("post")
        return {"performed": True}

    r2 = mom.launch_cuda_terrain_open_momentum_advection5(two, two, rrw_boundary_hook=rrw_hook,
                                                          post_divergence_hook=post_hook, **kw)
    torch.cuda.synchronize()
    assert seen == ["rrw", "post"] and r2.receipt["post_divergence"] == {"performed": True}
    for n in OUTS:
        _same(r2.divx if n == "divx" else two[n], (r1.divx if n == "divx" else one[n]).cpu().numpy(), n)


def test_bad_rrw_hook_receipt_refused():
    ni, nj, nk = 9, 8, 10
    a, m, _ = momentum_fixture(ni, nj, nk, 3)
    dev = _dev({**a, **m})
    with pytest.raises(ValueError, match="bcw"):
        mom.launch_cuda_terrain_open_momentum_advection5(
            dev, dev, ni=ni, nj=nj, nk=nk, nrk=1, dx=1.0, dy=1.0, dz=1.0,
            rrw_boundary_hook=lambda rrw, **k: {"performed": True})
    torch.cuda.synchronize()


def test_aliasing_refused():
    ni, nj, nk = 9, 8, 10
    a, m, _ = momentum_fixture(ni, nj, nk, 3)
    dev = _dev({**a, **m})
    dev["vten"] = dev["rrv"]
    with pytest.raises(ValueError, match="alias"):
        mom.launch_cuda_terrain_open_momentum_advection5(dev, dev, ni=ni, nj=nj, nk=nk, nrk=1, dx=1.0, dy=1.0,
                                                         dz=1.0)


@pytest.mark.parametrize("flat", [False, True])
@pytest.mark.parametrize("tag", ["momentum5_open_9x8x10", "momentum5_perx_8x9x9"])
def test_stretched_column_matches_oracle(flat, tag):
    """launch_cuda_gm1_child_stretched_momentum5 on a generated stretched
    column (20 m at the ground to 200 m at the top) against the oracle
    restatement, word for word, in the terrain branch and the flat column."""
    from gm1_b200.momentum import StretchedMomentumColumn, launch_cuda_gm1_child_stretched_momentum5
    from gm1_b200.vertical import build_vertical_levels
    from tests.test_oracle_momentum import _padded_rho0, load

    meta, a, _ = load(tag)
    ni, nj, nk = meta["ni"], meta["nj"], meta["nk"]
    spec = {10: (1100.0, 40.0, 700.0), 9: (990.0, 40.0, 590.0)}[nk]
    lv = build_vertical_levels(stretch_z=1, nk=nk, dz_m=100.0, ztop_m=spec[0], str_bot_m=spec[1], str_top_m=spec[2],
                               dz_bot_m=20.0, dz_top_m=200.0)
    rho0p = _padded_rho0(a["rho0_3d"], ni, nj, nk)
    rr0 = (np.float32(1.0) / a["rho0_3d"]).astype(np.float32)
    rdz = float(np.float32(1.0) / np.float32(100.0))
    a["divx"] = np.zeros((nk, nj, ni), np.float32)
    want = {k: v.copy() for k, v in a.items()}
    col = {"flat": flat, "rho0p": rho0p, "sigma": lv.sigma, "sigmaf": lv.sigmaf, "rds": lv.rds, "rdsf": lv.rdsf,
           "ztop": lv.ztop_m, "mh": lv.mh, "mf": lv.mf, "rr0": rr0, "rdz": rdz}
    if flat:
        for n in ("sigma", "sigmaf", "rds", "rdsf"):
            col[n] = None
    sides = tuple(meta["lateral_sides"])
    orc.momentum_advection5_column(want, col, ni=ni, nj=nj, nk=nk, dx=meta["dx"], dy=meta["dy"], lateral_sides=sides)
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in a.items()}
    t = lambda x: torch.from_numpy(np.array(x, dtype=np.float32)).cuda()  # noqa: E731
    vertical = (StretchedMomentumColumn(True, t(rho0p), mh=t(lv.mh), mf=t(lv.mf), rr0=t(rr0), rdz=rdz) if flat else
                StretchedMomentumColumn(False, t(rho0p), sigma=t(lv.sigma), sigmaf=t(lv.sigmaf), rds=t(lv.rds),
                                        rdsf=t(lv.rdsf), ztop=lv.ztop_m))
    launch_cuda_gm1_child_stretched_momentum5(d, d, vertical, ni=ni, nj=nj, nk=nk, nrk=1, dx=meta["dx"],
                                              dy=meta["dy"], divx=d["divx"], lateral_sides=sides)
    torch.cuda.synchronize()
    for n in ("uten", "vten", "wten", "rru", "rrv", "rrw", "divx"):
        got = d[n].cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want[n].view(np.uint32)), n
