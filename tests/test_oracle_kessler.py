"""Pins the Kessler oracle to the reference's own CPU twin
(cpu_gm1_kessler_driver_inplace) on golden fixtures: bit-exact where no
transcendental intervenes, the stated tolerances elsewhere."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import kessler as ko
from tests._golden import load_npz
from tests.kessler_common import assert_budgets_close, assert_fields_close

TAGS = ["kessler_eqt2_7x5x12", "kessler_eqt1_6x6x10"]


@pytest.mark.parametrize("tag", TAGS)
def test_kessler_oracle_matches_reference(tag):
    meta, inputs, out = load_npz(tag)
    a = {k: v.copy() for k, v in inputs.items()}
    it = np.zeros((meta["nk"], meta["nj"], meta["ni"]), np.uint32)
    nmax = ko.kessler_driver(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dx=meta["dx"], dy=meta["dy"],
                             dz=meta["dz"], dt=meta["dt"], eqtset=meta["eqtset"], iterations=it)
    assert nmax == meta["max_fall_substeps"]
    assert np.array_equal(it, out["satadj_iterations"])
    assert_fields_close(out, a)
    # pdefq and its budget meet no transcendental: bit-exact
    assert np.array_equal(a["asq"].view(np.uint64), out["asq"].view(np.uint64))
    assert_budgets_close(out["qbudget"], a["qbudget"])
