"""The stretched-column scalar advection oracle (restatement of the
reference's profile-bound advection texts,
src/cm1core/cuda_gm1_child_stretched_scalar.py:89-153, :262-352): on a
uniform column it reduces word for word to the uniform operator, which is
pinned to the reference's own twin; on a stretched column only the vertical
derivative (and, flat, the column's rr0 scale) changes.  The reference has
no CPU twin for the stretched family, so parity beyond the uniform limit is
pinned to this restatement only."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import advection as adv
from tests._golden import load_npz
from tests.test_oracle_advection import TAGS, advection_inputs


def _case(flat_uniform_rr0=False):
    meta, inputs, _ = load_npz(TAGS[0])
    h = advection_inputs(inputs, meta, "scalar")
    if flat_uniform_rr0:
        # a horizontally uniform base state and flat metrics
        h["rr0"][:] = h["rr0"][:, :1, :1]
        h["gz"][:] = np.float32(1.0)
    return meta, h


def _uniform(meta, h, nrk, sides):
    from gm1_b200.advection import scalar_open_boundary_code

    want = {k: v.copy() for k, v in h.items()}
    adv.scalar_advection5(want, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], nrk=nrk, dx=meta["dx"], dy=meta["dy"],
                          dz=meta["dz"], weps=meta["weps"]["scalar"], lateral_obc=scalar_open_boundary_code(sides))
    return want


def _column(meta, h, nrk, sides, flat, profile, rdz=0.0):
    from gm1_b200.advection import scalar_open_boundary_code

    got = {k: v.copy() for k, v in h.items()}
    adv.scalar_advection5_column(got, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], nrk=nrk, dx=meta["dx"],
                                 dy=meta["dy"], weps=meta["weps"]["scalar"], flat=flat, profile=profile, rdz=rdz,
                                 lateral_obc=scalar_open_boundary_code(sides))
    return got


@pytest.mark.parametrize("nrk", [1, 3])
@pytest.mark.parametrize("sides", [(2, 2, 2, 2), (1, 1, 1, 1)])
def test_uniform_terrain_column_is_the_uniform_operator(nrk, sides):
    meta, h = _case()
    nk = meta["nk"]
    rdsf = np.zeros(nk + 3, np.float32)
    rdsf[1:nk + 1] = np.float32(1.0) / np.float32(meta["dz"])
    want, got = _uniform(meta, h, nrk, sides), _column(meta, h, nrk, sides, False, rdsf)
    for n in ("tendency", "flux_x", "flux_y", "flux_z"):
        assert np.array_equal(want[n].view(np.uint32), got[n].view(np.uint32)), n


@pytest.mark.parametrize("nrk", [1, 3])
def test_uniform_flat_column_is_the_uniform_operator(nrk):
    meta, h = _case(flat_uniform_rr0=True)
    nk = meta["nk"]
    mh = np.ones(nk + 2, np.float32)
    rdz = float(np.float32(1.0) / np.float32(meta["dz"]))
    want, got = _uniform(meta, h, nrk, (2, 2, 2, 2)), _column(meta, h, nrk, (2, 2, 2, 2), True, mh, rdz)
    assert np.array_equal(want["tendency"].view(np.uint32), got["tendency"].view(np.uint32))


def test_stretched_column_changes_only_the_vertical_derivative():
    meta, h = _case()
    nk = meta["nk"]
    rng = np.random.default_rng(11)
    rdsf = np.zeros(nk + 3, np.float32)
    rdsf[1:nk + 1] = (np.float32(1.0) / np.float32(meta["dz"])) * rng.uniform(0.5, 2.0, nk).astype(np.float32)
    want, got = _uniform(meta, h, 1, (2, 2, 2, 2)), _column(meta, h, 1, (2, 2, 2, 2), False, rdsf)
    for n in ("flux_x", "flux_y", "flux_z"):
        assert np.array_equal(want[n].view(np.uint32), got[n].view(np.uint32)), n
    assert not np.array_equal(want["tendency"], got["tendency"])
