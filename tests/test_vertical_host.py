"""The library's vertical-coordinate host logic against the reference's own
generator (tests/golden/vertical_levels.json): build_vertical_levels forms
every profile word, rds/rdsf and the Fornberg weights on the host exactly as
build_vertical_levels of the reference does; derive_stretch_z1 gives the
reference's segment counts and coefficients; the reference's refusals are
refusals here."""

from __future__ import annotations

import numpy as np
import pytest

from gm1_b200.vertical import (PROFILES, StretchZ1Parameters, VerticalGridError, build_vertical_levels,
                               derive_stretch_z1, uniform_vertical_levels)
from tests._golden import load_json

G = load_json("vertical_levels.json")


def _levels(args):
    sz, nk, dz, ztop, sb, st, db, dt = args
    return build_vertical_levels(stretch_z=sz, nk=nk, dz_m=dz, ztop_m=ztop, str_bot_m=sb, str_top_m=st,
                                 dz_bot_m=db, dz_top_m=dt)


@pytest.mark.parametrize("name", sorted(G["cases"]))
def test_levels_are_the_reference_words(name):
    c = G["cases"][name]
    lv = _levels(c["args"])
    for f in PROFILES:
        assert np.array_equal(getattr(lv, f).view(np.uint32), np.array(c[f], np.uint32)), f
    for f in ("cgs", "cgt"):
        assert np.array_equal(np.array(getattr(lv, f), np.float32).view(np.uint32), np.array(c[f], np.uint32)), f
    assert lv.sha256 == c["sha256"]
    assert lv.ztop_m == c["ztop_m"]


@pytest.mark.parametrize("name", sorted(G["cases"]))
def test_derivation_is_the_reference_derivation(name):
    c = G["cases"][name]
    d = derive_stretch_z1(StretchZ1Parameters(*c["stretch_parameters"]))
    w = c["derived"]
    assert (d.nk1, d.nk2, d.nk3) == (w["nk1"], w["nk2"], w["nk3"])
    for f, g in (("nominal_dz_f32", "nominal"), ("c1_f32", "c1"), ("c2_f32", "c2")):
        assert np.float32(getattr(d, f)).view(np.uint32) == w[g], f


@pytest.mark.parametrize("name", sorted(G["refusals"]))
def test_reference_refusals_are_refused(name):
    with pytest.raises(VerticalGridError):
        _levels(G["refusals"][name]["args"])


def test_uniform_member_and_stretch_parameters_round_trip():
    u = uniform_vertical_levels(80, 250.0)
    assert u.uniform and u.ztop_m == 20000.0
    assert set(np.round(np.diff(u.zf[1:82]), 3)) == {250.0}
    c = G["cases"]["child_15km_nk75"]
    lv = _levels(c["args"])
    p = lv.stretch_parameters()
    assert [p.nk, p.dz, p.ztop, p.str_bot, p.str_top, p.dz_bot, p.dz_top] == c["stretch_parameters"]
    with pytest.raises(ValueError):
        derive_stretch_z1(StretchZ1Parameters(75, 100.0, 15000.0, 200.0, 7000.0, 30.0, 320.0))
