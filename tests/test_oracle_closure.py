"""The closure-input oracle (closure_oracle.c) against the reference's CPU
twins on seeded fixtures (tests/golden/calcdef_*.npz, moist_nm_*.npz, made by
make_golden.py closure).

Bars: calcdef (no transcendental) word for word; calcnm: the cell outputs
(temperature, qt, thv, qvci), the saturation mask and the branch counts word
for word, nm within NM_MAX_REL of max|nm| (logf/expf of the C library versus
NumPy's)."""

from __future__ import annotations

import json

import numpy as np
import pytest

from oracle import closure as orc
from tests._golden import GOLDEN

NM_MAX_REL = 5.0e-6
NM_EXACT = ("temperature", "qt", "thv", "qvci")


def load(tag):
    z = np.load(GOLDEN / f"{tag}.npz")
    meta = json.loads(str(z["meta"]))
    inputs = {k[3:]: z[k].copy() for k in z.files if k.startswith("in_")}
    outputs = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return meta, inputs, outputs


def nm_error(got, want) -> float:
    return float(np.max(np.abs(got.astype(np.float64) - want))) / float(np.max(np.abs(want)))


@pytest.mark.parametrize("tag", ["calcdef_9x7x8", "calcdef_12x6x10"])
def test_calcdef_oracle_bit_exact_vs_reference(tag):
    meta, a, want = load(tag)
    orc.calcdef(a, **{k: meta[k] for k in ("ni", "nj", "nk", "dx", "dy", "dz")})
    for n in ("defv", "defh"):
        assert np.array_equal(a[n].view(np.uint32), want[n].view(np.uint32)), n
    assert not np.any(a["defv"][0]) and not np.any(a["defh"][meta["nk"]])


@pytest.mark.parametrize("tag", ["moist_nm_8x6x14", "moist_nm_5x9x20"])
def test_moist_nm_oracle_vs_reference(tag):
    meta, a, want = load(tag)
    counts = orc.moist_nm(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dz=meta["dz"])
    assert counts == {k: meta[k] for k in ("saturated", "liquid", "mixed", "ice")}
    assert min(meta["liquid"], meta["mixed"], meta["ice"]) > 0  # every branch exercised
    for n in NM_EXACT:
        assert np.array_equal(a[n].view(np.uint32), want[n].view(np.uint32)), n
    assert np.array_equal(a["saturation_mask"], want["saturation_mask"])
    assert nm_error(a["nm"], want["nm"]) <= NM_MAX_REL
