"""The TKE-evolution oracle (tke_evolution_oracle.c) against the reference's
CPU twin cpu_tke_evolution_inplace on seeded terrain-lane inputs
(tests/golden/tke_evolution_*.npz, made by make_golden.py tkeevo): tketen
after turbt, the SHA-256 of every RK stage result, and the committed
tke3d/tkea, all word for word."""

from __future__ import annotations

import json

import numpy as np
import pytest

from oracle import tke_evolution as orc
from tests._golden import GOLDEN

PARAMS = ("ni", "nj", "nk", "dx", "dy", "dz", "dt")


def load(tag):
    z = np.load(GOLDEN / f"{tag}.npz")
    meta = json.loads(str(z["meta"]))
    return meta, {k[3:]: z[k].copy() for k in z.files if k.startswith("in_")}, \
        {k[4:]: z[k] for k in z.files if k.startswith("out_")}


@pytest.mark.parametrize("tag", ["tke_evolution_9x8x10", "tke_evolution_7x10x9"])
def test_tke_evolution_oracle_bit_exact_vs_reference(tag):
    meta, a, want = load(tag)
    hashes = orc.tke_evolution(a, **{k: meta[k] for k in PARAMS})
    assert hashes == meta["stage_sha256"]
    for n in ("tketen", "tke3d", "tkea"):
        assert np.array_equal(a[n].view(np.uint32), want[n].view(np.uint32)), n
    assert not np.any(a["tke3d"][0]) and not np.any(a["tke3d"][meta["nk"]])
