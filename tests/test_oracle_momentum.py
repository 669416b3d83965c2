"""The momentum-advection oracle (momentum_oracle.c) against the reference's
CPU twin cpu_terrain_open_momentum_advection5_inplace on seeded padded-lane
inputs in three lateral families (tests/golden/momentum5_*.npz, made by
make_golden.py momentum): rru, rrv, rrw, divx, uten, vten, wten word for
word.  Also the host-side contract of the mirror (no GPU needed)."""

from __future__ import annotations

import json

import numpy as np
import pytest

from gm1_b200 import momentum as mom
from oracle import momentum as orc
from tests._golden import GOLDEN

TAGS = ["momentum5_open_9x8x10", "momentum5_perx_8x9x9", "momentum5_walls_10x7x8"]
OUTS = ("uten", "vten", "wten", "rru", "rrv", "rrw", "divx")


def load(tag):
    z = np.load(GOLDEN / f"{tag}.npz")
    meta = json.loads(str(z["meta"]))
    return meta, {k[3:]: z[k].copy() for k in z.files if k.startswith("in_")}, \
        {k[4:]: z[k] for k in z.files if k.startswith("out_")}


@pytest.mark.parametrize("tag", TAGS)
def test_momentum_oracle_bit_exact_vs_reference(tag):
    meta, a, want = load(tag)
    a["divx"] = np.zeros((meta["nk"], meta["nj"], meta["ni"]), np.float32)
    orc.momentum_advection5(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dx=meta["dx"], dy=meta["dy"],
                            dz=meta["dz"], lateral_sides=tuple(meta["lateral_sides"]))
    for n in OUTS:
        assert np.array_equal(a[n].view(np.uint32), want[n].view(np.uint32)), n


def test_lateral_family_words():
    assert mom.momentum_open_boundary_code((2, 2, 2, 2)) == 0x2222
    assert mom.momentum_open_boundary_code((3, 4, 1, 1)) == 3 | 4 << 4 | 1 << 8 | 1 << 12
    assert mom.momentum_advection5_counts(9, 8, 10, (1, 1, 2, 2)) == (10 * 8 * 10, 10 * 7 * 9, 9 * 8 * 9)
    assert mom.momentum_advection5_counts(9, 8, 10) == (10 * 8 * 8, 10 * 7 * 9, 9 * 8 * 9)
    f = mom.momentum_boundary_faces((1, 1, 2, 3))
    assert f["advu_faces_one_based"] == [1, "ni+1"] and f["advv_rows_one_based"] == [2, "nj"]
    assert f["inflow_edits_on"] == ["south"]


@pytest.mark.parametrize("sides", [(1, 2, 2, 2), (2, 2, 3, 1), (0, 2, 2, 2), (2, 2, 2), (True, 2, 2, 2)])
def test_lateral_sides_refused(sides):
    with pytest.raises(ValueError):
        mom.momentum_lateral_sides(sides)


def test_selection_refused_by_field():
    with pytest.raises(ValueError, match="advwenov"):
        mom.validate_momentum_advection5_selection(mom.MomentumAdvection5Selection(advwenov=1))
    with pytest.raises(ValueError, match="hadvordrv"):
        mom.validate_momentum_advection5_selection(mom.MomentumAdvection5Selection(hadvordrv=6))
    with pytest.raises(TypeError):
        mom.validate_momentum_advection5_selection(None)


def test_launcher_refuses_before_touching_a_device():
    kw = dict(ni=9, nj=8, nk=10, nrk=1, dx=400.0, dy=350.0, dz=180.0)
    with pytest.raises(ValueError, match="nrk"):
        mom.launch_cuda_terrain_open_momentum_advection5({}, {}, **{**kw, "nrk": 4})
    with pytest.raises(ValueError, match="nk"):
        mom.launch_cuda_terrain_open_momentum_advection5({}, {}, **{**kw, "nk": 7})
    with pytest.raises(ValueError, match="dx"):
        mom.launch_cuda_terrain_open_momentum_advection5({}, {}, **{**kw, "dx": float("nan")})
    with pytest.raises(TypeError, match="post_divergence_hook"):
        mom.launch_cuda_terrain_open_momentum_advection5({}, {}, post_divergence_hook=3, **kw)
    with pytest.raises(ValueError, match="periodic"):
        mom.launch_cuda_terrain_open_momentum_advection5({}, {}, lateral_sides=(1, 2, 2, 2), **kw)
    meta, a, _ = load(TAGS[0])
    import torch
    cpu = {k: torch.from_numpy(v) for k, v in a.items()}
    with pytest.raises(TypeError, match="CUDA"):
        mom.launch_cuda_terrain_open_momentum_advection5(cpu, cpu, **kw)


def _padded_rho0(rho0, ni, nj, nk):
    """(nk+2, nj+6, ni+6) base density whose halo repeats the edge column /
    row (the clamp the uniform operator applies)."""
    p = np.zeros((nk + 2, nj + 6, ni + 6), np.float32)
    p[1:nk + 1, 3:nj + 3, 3:ni + 3] = rho0
    p[1:nk + 1, 3:nj + 3, :3] = rho0[:, :, :1]
    p[1:nk + 1, 3:nj + 3, ni + 3:] = rho0[:, :, -1:]
    p[:, :3, :] = p[:, 3:4, :]
    p[:, nj + 3:, :] = p[:, nj + 2:nj + 3, :]
    return p


def test_uniform_terrain_column_is_the_uniform_operator():
    """The stretched momentum (restatement of the reference's profile-bound
    text, cuda_gm1_child_stretched_momentum.py:56-200) on the uniform column's
    own sigma/sigmaf/rds/rdsf words and a clamped-halo padded density is the
    twin-pinned uniform operator word for word."""
    from gm1_b200.vertical import uniform_vertical_levels

    meta, a, _ = load(TAGS[0])
    ni, nj, nk = meta["ni"], meta["nj"], meta["nk"]
    a["divx"] = np.zeros((nk, nj, ni), np.float32)
    b = {k: v.copy() for k, v in a.items()}
    orc.momentum_advection5(a, ni=ni, nj=nj, nk=nk, dx=meta["dx"], dy=meta["dy"], dz=meta["dz"],
                            lateral_sides=tuple(meta["lateral_sides"]))
    lv = uniform_vertical_levels(nk, meta["dz"])
    col = {"flat": False, "rho0p": _padded_rho0(b["rho0_3d"], ni, nj, nk), "sigma": lv.sigma, "sigmaf": lv.sigmaf,
           "rds": lv.rds, "rdsf": lv.rdsf, "ztop": lv.ztop_m}
    orc.momentum_advection5_column(b, col, ni=ni, nj=nj, nk=nk, dx=meta["dx"], dy=meta["dy"],
                                   lateral_sides=tuple(meta["lateral_sides"]))
    for n in OUTS:
        assert np.array_equal(a[n].view(np.uint32), b[n].view(np.uint32)), n
