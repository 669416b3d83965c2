"""The CM1 limits oracle (limits_oracle.c) against the reference's own
functions (tests/golden/limits_courant.npz, made by make_golden.py limits):
the small-step bound, the diagnostic substep count and the scalar Courant
number exactly (binary64), the domain Courant number word for word
(binary32), NaN and inf levels included."""

from __future__ import annotations

import json

import numpy as np
import pytest

from oracle import limits as orc
from tests._golden import GOLDEN

F = np.float32


def _cases():
    z = np.load(GOLDEN / "limits_courant.npz")
    table = json.loads(str(z["table"]))
    tags = sorted({k.split("_", 1)[0] for k in z.files if k != "table"})
    return z, table, tags


def factors(meta):
    return tuple(float(F(F(F(0.5) * F(meta["dt"])) * F(1.0 / meta[d]))) for d in ("dx", "dy", "dz"))


def test_scalar_limits_match_reference_table():
    _, table, _ = _cases()
    assert len(table) == 42
    for row in table:
        assert orc.small_step_limit(row["dx"], row["dy"]) == row["limit"]
        assert orc.diagnostic_substeps(row["dt"], row["dx"], row["dy"]) == row["nsound"]
        got = orc.advective_courant(row["dt"], row["dx"], row["dy"], row["dz"], row["u"], row["v"], row["w"])
        assert got == row["courant"]


@pytest.mark.parametrize("tag", ["a", "b", "c", "d", "e"])
def test_domain_courant_matches_reference(tag):
    z, _, _ = _cases()
    meta = json.loads(str(z[f"{tag}_meta"]))
    got, levels = orc.courant_max(z[f"{tag}_u"], z[f"{tag}_v"], z[f"{tag}_w"], z[f"{tag}_uh"], z[f"{tag}_vh"],
                                  z[f"{tag}_mh"], *factors(meta))
    want = meta["courant"]
    assert (got == want) or (np.isinf(got) and np.isinf(want))
    assert levels.shape == (meta["nz"],)
