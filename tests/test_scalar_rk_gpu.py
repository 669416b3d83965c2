"""Parity of the CUDA scalar/moisture RK pieces (through the C ABI) with the
reference's CPU twins (golden vectors) and the oracle: every word identical."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.scalar_rk import compose_scalar_moist_rk_stage, pdef_direction, theta_transport_scalar
from oracle import rk
from tests._golden import load_npz
from tests.test_oracle_rk import TAGS, bits_equal

pytestmark = pytest.mark.gpu


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("tag", TAGS)
def test_pack_and_compose_bit_exact_vs_reference(tag):
    meta, a, out = load_npz(tag)
    pad = dev(a["theta_pad"])
    theta_transport_scalar(dev(a["th0"]), dev(a["th3d"]), pad, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"])
    torch.cuda.synchronize()
    assert bits_equal(pad.cpu().numpy(), out["theta_pad"])
    for nrk in (1, 2, 3):
        tc = torch.zeros_like(dev(a["theta_a"]))
        qc = torch.zeros_like(dev(a["q_a"]))
        compose_scalar_moist_rk_stage(dev(a["theta_a"]), dev(a["q_a"]), dev(a["theta_held"]), dev(a["q_held"]),
                                      dev(a["theta_divterm"]), dev(a["theta_adv"]), dev(a["q_adv"]), tc, qc,
                                      nrk=nrk, dt=meta["dt"])
        torch.cuda.synchronize()
        assert bits_equal(tc.cpu().numpy(), out[f"theta_cur_{nrk}"])
        assert bits_equal(qc.cpu().numpy(), out[f"q_cur_{nrk}"])


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_pdef_direction_bit_exact_vs_reference(tag, axis):
    meta, a, out = load_npz(tag)
    d = dev(a["pd_directional"])
    cand = torch.zeros_like(d)
    pdef_direction(dev(a["pd_scalar_a"]), dev(a["pd_scalar_padded"]), dev(a["pd_rho0"]), dev(a["pd_gz"]),
                   dev(a["pd_rgz"]), dev(a[f"pd_flux_{axis}"]), d, cand, axis=axis, dt=meta["pdef_dt"],
                   spacing=meta["spacing"][axis])
    torch.cuda.synchronize()
    assert bits_equal(cand.cpu().numpy(), out[f"pd_candidate_{axis}"])
    assert bits_equal(d.cpu().numpy(), out[f"pd_directional_{axis}"])


@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_pdef_large_matches_oracle(axis):
    from tests.golden.make_golden import rk_fixture

    ni, nj, nk = 130, 70, 40
    a = rk_fixture(ni, nj, nk, 555)
    want_d = a["pd_directional"].copy()
    want_c = np.zeros_like(want_d)
    spacing = {"x": 1000.0, "y": 900.0, "z": 250.0}[axis]
    rk.pdef_direction(a["pd_scalar_a"], a["pd_scalar_padded"], a["pd_rho0"], a["pd_gz"], a["pd_rgz"],
                      a[f"pd_flux_{axis}"], want_d, want_c, axis=axis, dt=1.5, spacing=spacing)
    d = dev(a["pd_directional"])
    cand = torch.zeros_like(d)
    pdef_direction(dev(a["pd_scalar_a"]), dev(a["pd_scalar_padded"]), dev(a["pd_rho0"]), dev(a["pd_gz"]),
                   dev(a["pd_rgz"]), dev(a[f"pd_flux_{axis}"]), d, cand, axis=axis, dt=1.5, spacing=spacing)
    torch.cuda.synchronize()
    assert bits_equal(cand.cpu().numpy(), want_c) and bits_equal(d.cpu().numpy(), want_d)
