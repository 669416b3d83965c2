"""The vertical-coordinate oracle against the reference's own generator
(tests/golden/vertical_levels.json, made by make_golden.py vertical from
build_vertical_levels / derive_stretch_z1): every profile word, rds/rdsf,
the Fornberg weights and the derived segment counts for stretch_z 0 and 1,
and the reference's refusals.  The 15 km child's words also reproduce the
digests the reference seals for that grid (stretch_z1_child_15km.py)."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle import vertical as orv
from tests._golden import load_json

G = load_json("vertical_levels.json")


def _f32(words):
    return np.array(words, dtype=np.uint32).view(np.float32)


@pytest.mark.parametrize("name", sorted(G["cases"]))
def test_oracle_levels_match_reference_words(name):
    c = G["cases"][name]
    sz, nk, dz, ztop, sb, st, db, dt = c["args"]
    rc, out = orv.vertical_levels(sz, nk, dz, ztop, sb, st, db, dt)
    assert rc == 0
    for f in orv.PROFILES + ("cgs", "cgt"):
        assert np.array_equal(out[f].view(np.uint32), np.array(c[f], np.uint32)), f


@pytest.mark.parametrize("name", sorted(G["cases"]))
def test_oracle_derivation_matches_reference(name):
    c = G["cases"][name]
    rc, d = orv.derive_stretch_z1(*c["stretch_parameters"])
    assert rc == 0
    want = c["derived"]
    assert (d.nk1, d.nk2, d.nk3) == (want["nk1"], want["nk2"], want["nk3"])
    for f in ("nominal", "c1", "c2"):
        assert np.float32(getattr(d, f)).view(np.uint32) == want[f], f


def test_child_words_reproduce_the_reference_seal():
    c = G["cases"]["child_15km_nk75"]
    for f, h in G["sealed_child_15km_profile_sha256"].items():
        assert hashlib.sha256(_f32(c[f]).astype("<f4").tobytes()).hexdigest() == h, f


@pytest.mark.parametrize("name", sorted(G["refusals"]))
def test_oracle_refuses_what_the_reference_refuses(name):
    sz, nk, dz, ztop, sb, st, db, dt = G["refusals"][name]["args"]
    rc, _ = orv.vertical_levels(sz, nk, dz, ztop, sb, st, db, dt)
    assert rc < 0
