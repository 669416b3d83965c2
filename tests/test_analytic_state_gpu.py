"""The library's analytic initial state (libgm1b.so through gm1_b200.analytic_state)
against CM1 r21.1's own output, the reference's sealed words and the oracle.

Bars: the base column and the wind profile are host binary32 arithmetic with
the C library's powf/expf/cosf/sinf, so they are word-identical to the oracle
and to CM1 (th0, qv0, pi0; prs0 within 2 ulp of CM1, identical to the
oracle).  The bubble is a CUDA kernel: its support (beta < 1, from correctly
rounded divides and sqrtf) is bit-identical to the oracle; inside it the
device cosf may differ from the C library's by an ulp or two, so values agree
within 4 ulp of the amplitude (|d| <= 4 * 2^-23 * amp)."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest
import torch

from gm1_b200.analytic_state import (
    WarmBubbleControls,
    analytic_shear_u,
    analytic_shear_v,
    build_theta_perturbation,
    weisman_klemp_column,
    weisman_klemp_column_with_iterations,
)
from oracle import initial as orc
from tests._golden import load_json
from tests.test_oracle_initial import deck_heights, ulps, words

pytestmark = pytest.mark.gpu


def test_wk_column_matches_cm1_and_oracle_words():
    record = load_json("wk_cm1_nz40.json")
    z = deck_heights(40, 500.0)
    col = weisman_klemp_column(z, 1)
    for name, got in (("th0", col.theta_k), ("qv0", col.qv_kg_per_kg), ("pi0", col.pi)):
        assert words(got) == record["cm1_words"][name], name
    assert int(ulps(col.pressure_pa, record["cm1_words"]["prs0"]).max()) <= 2
    for name, got in (("qv0", col.qv_kg_per_kg), ("pi0", col.pi)):
        assert hashlib.sha256(got.astype("<f4").tobytes()).hexdigest() == record["sealed_sha256"][name]
    want = orc.wk_column(z, 1, 20)
    for name, got in (("th0", col.theta_k), ("qv0", col.qv_kg_per_kg), ("thv0", col.theta_v_k), ("pi0", col.pi),
                      ("prs0", col.pressure_pa), ("t0", col.temperature_k), ("rh0", col.relative_humidity)):
        assert words(got) == words(want[name]), name


@pytest.mark.parametrize("nz,dz,imoist", [(64, 250.0, 1), (48, 400.0, 0), (80, 250.0, 1)])
def test_wk_column_matches_oracle_on_other_decks(nz, dz, imoist):
    z = deck_heights(nz, dz)
    col = weisman_klemp_column_with_iterations(z, imoist, 20)
    want = orc.wk_column(z, imoist, 20)
    assert words(col.pi) == words(want["pi0"]) and words(col.qv_kg_per_kg) == words(want["qv0"])
    assert words(col.pressure_pa) == words(want["prs0"]) and words(col.theta_k) == words(want["th0"])


def test_wk_surface_qv_rule():
    col = weisman_klemp_column(deck_heights(40, 500.0), 1)
    assert col.surface_qv_kg_per_kg([1.875, -1.25, 0.375]) == np.float32(0.014)
    dry = weisman_klemp_column(deck_heights(40, 500.0), 0)
    assert dry.surface_qv_kg_per_kg([1.875, -1.25, 0.375]) == 0.0


def test_analytic_shear_matches_oracle_bit_for_bit():
    z = np.arange(-500.0, 20000.0 + 1.0, 12.5, dtype=np.float32)
    u_want, v_want = orc.analytic_shear(z, z)
    assert words(analytic_shear_u(z)) == words(u_want)
    assert words(analytic_shear_v(z)) == words(v_want)


@pytest.mark.parametrize("ng", [0, 1, 3])
def test_theta_bubble_kernel_matches_oracle(ng):
    ni, nj, nk = 37, 29, 40
    xh = (np.arange(ni, dtype=np.float32) - np.float32(18.0)) * np.float32(1000.0)
    yh = (np.arange(nj, dtype=np.float32) - np.float32(14.0)) * np.float32(1000.0)
    zh = deck_heights(nk, 500.0)
    ctl = WarmBubbleControls(center_x_m=0.0, center_y_m=0.0, center_z_agl_m=1400.0, horizontal_radius_m=10000.0,
                             vertical_radius_m=1400.0, amplitude_k=2.0)
    want = orc.theta_bubble(xh, yh, zh, xc=0.0, yc=0.0, zc=1400.0, hrad=10000.0, zrad=1400.0, amp=2.0)
    gz = 1 if ng else 0
    sentinel = -7.0
    tha = torch.full((nk + 2 * gz, nj + 2 * ng, ni + 2 * ng), sentinel, dtype=torch.float32, device="cuda")
    dev = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    build_theta_perturbation(tha, ctl, xh=dev(xh), yh=dev(yh), zh=dev(zh), ni=ni, nj=nj, nk=nk, ng=ng)
    torch.cuda.synchronize()
    got_full = tha.cpu().numpy()
    got = got_full[gz:gz + nk, ng:ng + nj, ng:ng + ni]
    assert np.array_equal(got != 0.0, want != 0.0)  # identical support
    assert float(np.max(np.abs(got - want))) <= 4 * 2.0**-23 * 2.0
    halo = np.ones(got_full.shape, bool)
    halo[gz:gz + nk, ng:ng + nj, ng:ng + ni] = False
    assert np.all(got_full[halo] == sentinel)  # halo words untouched


def test_refusals():
    with pytest.raises(ValueError, match="strictly increasing"):
        weisman_klemp_column(np.array([500.0, 400.0], np.float32), 1)
    with pytest.raises(ValueError, match="imoist"):
        weisman_klemp_column(deck_heights(4, 500.0), 3)
    with pytest.raises(ValueError, match="iteration"):
        weisman_klemp_column_with_iterations(deck_heights(4, 500.0), 1, 0)
    with pytest.raises(ValueError, match="nk>=1"):
        weisman_klemp_column(np.zeros(0, np.float32), 1)
