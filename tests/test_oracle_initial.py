"""The analytic initial-state oracle (init_oracle.c) pinned against CM1 r21.1's
own output and the reference's sealed binary32 words.

Pins (tests/golden/wk_cm1_nz40.json, made by make_golden.py wk):
  * CM1 r21.1 supercell run, isnd=5, nz=40, dz=500 m: th0, qv0 and pi0 word
    for word; prs0 within 2 ulp (CM1's written prs0 is not p00*pi0**(cp/rd)
    of its own pi0 in any binary32/binary64 evaluation order tried; the
    reference restates base.F:421-423 as that expression,
    rust/cm1-state/src/storm_initialization.rs:273-276, and so does this
    oracle).
  * the reference's sealed SHA-256 digests of the qv0 and pi0 words
    (storm_initialization.rs, hydrostatic_fixed_point_is_settled_at_the_source_iteration_count).
  * the reference's hand-evaluated source checks of the wind profile at named
    heights (storm_initialization.rs, analytic_wind_profile_matches_hand_evaluated_source_at_named_heights).
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle import initial as orc
from tests._golden import load_json

F = np.float32


def deck_heights(nz: int, dz: float) -> np.ndarray:
    # 0.5*(dz*k + dz*(k+1)) in binary32 (storm_initialization.rs:858-862)
    return np.array([F(0.5) * (F(dz) * F(k) + F(dz) * F(k + 1)) for k in range(nz)], dtype=np.float32)


def words(a: np.ndarray) -> list[str]:
    return [f"{int(w):08x}" for w in np.asarray(a, dtype=np.float32).view(np.uint32)]


def ulps(a: np.ndarray, b_words: list[str]) -> np.ndarray:
    b = np.array([int(w, 16) for w in b_words], dtype=np.uint32).view(np.int32).astype(np.int64)
    return np.abs(np.asarray(a, np.float32).view(np.int32).astype(np.int64) - b)


@pytest.fixture(scope="module")
def record():
    return load_json("wk_cm1_nz40.json")


@pytest.fixture(scope="module")
def column():
    return orc.wk_column(deck_heights(40, 500.0), 1, 20)


def test_wk_column_matches_cm1_output_words(record, column):
    for name in ("th0", "qv0", "pi0"):
        assert words(column[name]) == record["cm1_words"][name], name
    assert record["cm1_pi0_column_derived_variant"] == record["cm1_words"]["pi0"]
    assert int(ulps(column["prs0"], record["cm1_words"]["prs0"]).max()) <= 2


def test_wk_column_matches_sealed_reference_digests(record, column):
    for name in ("qv0", "pi0"):
        digest = hashlib.sha256(column[name].astype("<f4").tobytes()).hexdigest()
        assert digest == record["sealed_sha256"][name], name


def test_wk_surface_words():
    pi, qv, thv = orc.wk_surface()
    assert pi == F(1.0)
    assert qv > 0.0 and thv > F(300.0)


def test_wk_named_heights_and_cap():
    z = np.array([1000.0, 3000.0, 6000.0, 11999.0, 12000.0, 18000.0], dtype=np.float32)
    c = orc.wk_column(z, 1, 20)
    assert abs(c["th0"][2] - F(318.07928)) < 1.0e-3
    assert c["th0"][4] == F(343.0)
    assert abs(c["th0"][5] - F(451.467)) < 1.0e-2
    assert c["th0"][3] < F(343.0)
    assert c["qv0"][0] == F(0.014)


def test_wk_fixed_point_settled_at_twenty_iterations():
    z = deck_heights(40, 500.0)
    twenty = orc.wk_column(z, 1, 20)
    for extra in (21, 40):
        more = orc.wk_column(z, 1, extra)
        for name in ("qv0", "pi0", "prs0", "thv0", "rh0"):
            assert words(more[name]) == words(twenty[name]), (name, extra)
    one = orc.wk_column(z, 1, 1)
    assert words(one["qv0"]) != words(twenty["qv0"])
    assert np.all(np.diff(twenty["pi0"]) < 0) and np.all(np.diff(twenty["prs0"]) < 0)


def test_wk_dry_column_has_no_vapour():
    dry = orc.wk_column(deck_heights(40, 500.0), 0, 20)
    assert not np.any(dry["qv0"])


def test_wk_oracle_refusals():
    with pytest.raises(ValueError):
        orc.wk_column(np.array([500.0, 500.0], np.float32))
    with pytest.raises(ValueError):
        orc.wk_column(deck_heights(4, 500.0), 2)
    with pytest.raises(ValueError):
        orc.wk_column(deck_heights(4, 500.0), 1, 0)


def test_analytic_shear_named_heights():
    pi = F(np.pi)
    low = np.array([0.0, 500.0, 1000.0, 1999.0, 2000.0], np.float32)
    u, v = orc.analytic_shear(low, low)
    for q, z in enumerate(low):
        angle = F(F(F(90.0) * F(z / F(2000.0))) * F(pi / F(180.0)))
        # the C library's cosf/sinf against binary64: within a few binary32 ulps of 7
        assert abs(u[q] - (7.0 - 7.0 * np.cos(np.float64(angle)))) < 2e-6
        assert abs(v[q] - 7.0 * np.sin(np.float64(angle))) < 2e-6
    high = np.array([2001.0, 3000.0, 4000.0, 6000.0, 9000.0], np.float32)
    u, v = orc.analytic_shear(high, high)
    for q, z in enumerate(high[:4]):
        assert u[q] == F(F(7.0) + F(F(z - F(2000.0)) * F(24.0)) / F(4000.0))
    assert u[4] == F(31.0) and np.all(v == F(7.0))
    u0, v0 = orc.analytic_shear(np.zeros(1, np.float32), np.zeros(1, np.float32))
    assert u0[0] == 0.0 and v0[0] == 0.0


def test_theta_bubble_shape():
    xh = (np.arange(24, dtype=np.float32) - F(11.5)) * F(1000.0)
    tha = orc.theta_bubble(xh, xh, deck_heights(40, 500.0), xc=0.0, yc=0.0, zc=1400.0, hrad=10000.0,
                           zrad=1400.0, amp=1.0)
    assert tha.shape == (40, 24, 24)
    assert float(tha.max()) <= 1.0 and float(tha.min()) == 0.0
    assert np.array_equal(tha, tha[:, ::-1, :]) and np.array_equal(tha, tha[:, :, ::-1])
    assert not np.any(tha[8:])  # above zc + zrad
