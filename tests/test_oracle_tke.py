"""Pins the SGS/TKE oracle to the reference's own CPU twin
(cpu_sgs_tke_inplace) on golden fixtures under the stated tolerance."""

from __future__ import annotations

import pytest

from oracle import tke as to
from tests._golden import load_npz
from tests.tke_common import assert_sgs_close

TAGS = ["sgs_tke_9x7x12", "sgs_tke_6x8x10"]


@pytest.mark.parametrize("tag", TAGS)
def test_sgs_tke_oracle_matches_reference(tag):
    meta, inputs, out = load_npz(tag)
    a = {k: v.copy() for k, v in inputs.items()}
    clipped = to.sgs_tke(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dx=meta["dx"], dy=meta["dy"], dz=meta["dz"])
    assert clipped == meta["clipped"]
    assert_sgs_close(out, a)


def test_sgs_constants_match_reference():
    meta, _, _ = load_npz(TAGS[0])
    assert to.sgs_constants() == meta["constants"]
