"""Pins the Kessler large-step oracle (held-rate remove/snapshot, pre-physics
EOS, driver, held recapture) to the reference's CPU twin
cpu_gm1_kessler_large_step_inplace on golden fixtures, under the Kessler
tolerances (tests/kessler_common.py); the held rates are compared as the
state increments rate * dt they stand for, on the scale of the full field."""

from __future__ import annotations

import json

import numpy as np
import pytest

from oracle import kessler as ko
from tests._golden import GOLDEN
from tests.kessler_common import MAX_ABS_REL, assert_fields_close, full_variable

TAGS = ["kessler_large_step_eqt2_7x5x12", "kessler_large_step_eqt1_6x6x10"]
HELD_OF = {"qpten": "pp3d", "qtten": "th3d", "qvten": "qv", "qcten": "qc"}


def load(tag):
    z = np.load(GOLDEN / f"{tag}.npz")
    meta = json.loads(str(z["meta"]))
    pick = lambda p: {k[len(p):]: z[k].copy() for k in z.files if k.startswith(p)}  # noqa: E731
    return meta, pick("in_"), pick("held_in_"), pick("out_"), pick("held_out_")


def assert_held_close(want_held, got_held, want_fields, dt):
    for h, f in HELD_OF.items():
        scale = float(np.max(np.abs(full_variable(f, want_fields))))
        err = float(np.max(np.abs(want_held[h].astype(np.float64) - got_held[h]))) * dt
        assert err <= MAX_ABS_REL * scale, (h, err, scale)


@pytest.mark.parametrize("tag", TAGS)
def test_large_step_oracle_matches_reference(tag):
    meta, a, held, want, want_held = load(tag)
    nmax = ko.kessler_large_step(a, held, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dx=meta["dx"], dy=meta["dy"],
                                 dz=meta["dz"], dt=meta["dt"], eqtset=meta["eqtset"])
    assert nmax == meta["max_fall_substeps"]
    assert_fields_close(want, a)
    assert np.array_equal(a["rr"].view(np.uint32), a["rr"].view(np.uint32))
    if meta["eqtset"] == 2:
        assert_held_close(want_held, held, want, meta["dt"])
    else:
        for n in HELD_OF:
            assert np.array_equal(held[n], want_held[n])
