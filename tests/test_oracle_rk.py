"""Pins the scalar/moisture RK oracle to the reference's own CPU twins
(theta packing, RK composition at nrk 1..3, pdef on each axis) word for word."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import rk
from tests._golden import load_npz

TAGS = ["rk_11x9x8", "rk_7x12x10"]


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


@pytest.mark.parametrize("tag", TAGS)
def test_theta_pack_and_compose_match_reference(tag):
    meta, a, out = load_npz(tag)
    pad = a["theta_pad"].copy()
    rk.theta_pack(a["th0"], a["th3d"], pad, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"])
    assert bits_equal(pad, out["theta_pad"])
    for nrk in (1, 2, 3):
        tc = np.zeros_like(a["theta_a"])
        qc = np.zeros_like(a["q_a"])
        rk.compose(a["theta_a"], a["q_a"], a["theta_held"], a["q_held"], a["theta_divterm"], a["theta_adv"],
                   a["q_adv"], tc, qc, nrk=nrk, dt=meta["dt"])
        assert bits_equal(tc, out[f"theta_cur_{nrk}"]) and bits_equal(qc, out[f"q_cur_{nrk}"]), nrk


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_pdef_direction_matches_reference(tag, axis):
    meta, a, out = load_npz(tag)
    d = a["pd_directional"].copy()
    cand = np.zeros_like(d)
    rk.pdef_direction(a["pd_scalar_a"], a["pd_scalar_padded"], a["pd_rho0"], a["pd_gz"], a["pd_rgz"],
                      a[f"pd_flux_{axis}"], d, cand, axis=axis, dt=meta["pdef_dt"], spacing=meta["spacing"][axis])
    assert bits_equal(cand, out[f"pd_candidate_{axis}"])
    assert bits_equal(d, out[f"pd_directional_{axis}"])
    assert not bits_equal(d, a["pd_directional"])  # the repair fired
