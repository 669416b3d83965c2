"""The oracle's restatement of the final-RK dry-air mass correction against
the reference's own CPU twin (golden apmasscon_*.npz from
tests/golden/make_golden.py apmasscon): the binary64 ledgers mass2 and the
Exner sum and the binary64 correction equal (the same serial order), pp3d
word-identical, prs and rho within 2 ulp (powf: the C library's against
NumPy's), and the initial ledger mass1 of the starting state equal."""

from __future__ import annotations

import json

import numpy as np
import pytest

from oracle import kessler as oks
from tests._golden import GOLDEN


def _ulps(a: np.ndarray, b: np.ndarray) -> int:
    return int(np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64)).max())


@pytest.mark.parametrize("tag", ["apmasscon_9x7x12", "apmasscon_13x6x10"])
def test_oracle_matches_the_reference_twin(tag):
    from tests.golden.make_golden import APMASSCON_CASES, apmasscon_fixture  # noqa: PLC0415

    z = np.load(GOLDEN / f"{tag}.npz")
    meta = json.loads(str(z["meta"]))
    ni, nj, nk = meta["ni"], meta["nj"], meta["nk"]
    start = apmasscon_fixture(ni, nj, nk, APMASSCON_CASES[tag][3])
    assert oks.dry_mass(start["rho"], start["ruh"], start["rvh"], start["rmh"], ni=ni, nj=nj, nk=nk) == meta["mass1"]
    a = {n: z[f"in_{n}"].copy() for n in oks.APMASSCON_NAMES}
    d = oks.apmasscon(a, ni=ni, nj=nj, nk=nk, mass1=meta["mass1"])
    assert d[0] == meta["mass2"] and d[1] == meta["pressure_sum"] and d[3] == meta["mass1"]
    assert np.float32(d[2]) == np.float32(meta["correction"]) and meta["correction"] != 0.0
    assert np.array_equal(a["pp3d"].view(np.uint32), z["out_pp3d"].view(np.uint32))
    for n in ("prs", "rho"):
        assert _ulps(a[n], z[f"out_{n}"]) <= 2, n
