"""The terrain/open acoustic-stage oracle (terrain_open_oracle.c) against
the reference's CPU twin cpu_psolver3_terrain_open_stage_inplace
(tests/golden/tos_*.npz, made by make_golden.py terrainopen): every one of
the 45 arrays after each of the three RK stages, the cadence, each of the
eight ablations and non-default alph/kdiv, word for word."""

from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

from oracle import terrain_open as orc
from tests._golden import GOLDEN

TAGS = ["tos_reftest_5x4x5", "tos_seeded_9x7x8", "tos_seeded_6x10x6"]
PARAMS = ("ni", "nj", "nk", "dt", "nsound", "dx", "dy", "dz")


def load(tag):
    z = np.load(GOLDEN / f"{tag}.npz")
    meta = json.loads(str(z["meta"]))
    a = {k[3:]: z[k].copy() for k in z.files if k.startswith("in_")}
    m = {k[7:]: z[k].copy() for k in z.files if k.startswith("metric_")}
    want = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return meta, a, m, want


def digest(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x).astype("<f4", copy=False).tobytes()).hexdigest()


def digests(a):
    return {n: digest(a[n]) for n in orc.ARRAY_NAMES}


def _mismatch(got, want):
    return sorted(n for n in want if got[n] != want[n])


@pytest.mark.parametrize("tag", TAGS)
def test_three_stages_bit_exact_vs_reference(tag):
    meta, a, m, want = load(tag)
    p = {k: meta[k] for k in PARAMS}
    for stage in meta["stages"]:
        d = orc.terrain_open_stage(a, m, nrk=stage["nrk"], **p)
        assert (d.nloop, d.dts_f32) == (stage["nloop"], stage["dts_f32"])
        assert d.max_tridiagonal_residual == pytest.approx(stage["max_tridiagonal_residual"], rel=0, abs=0)
        assert _mismatch(digests(a), stage["digests"]) == [], f"nrk={stage['nrk']}"
    for n in orc.ARRAY_NAMES:
        assert np.array_equal(a[n].view(np.uint32), want[n].view(np.uint32)), n


def test_reference_cadence_and_residual_bound():
    meta, *_ = load("tos_reftest_5x4x5")
    assert [s["nloop"] for s in meta["stages"]] == [2, 3, 6]
    assert max(s["max_tridiagonal_residual"] for s in meta["stages"]) < 1.0e-5


@pytest.mark.parametrize("name", list(orc.ABLATION_BITS))
def test_each_ablation_bit_exact_vs_reference(name):
    meta, a, m, _ = load("tos_reftest_5x4x5")
    p = {k: meta[k] for k in PARAMS}
    orc.terrain_open_three_stage(a, m, ablations=orc.ablation_mask(**{name: False}), **p)
    assert _mismatch(digests(a), meta["ablations"][name]) == []
    assert meta["ablations"][name]["u3d"] != meta["stages"][2]["digests"]["u3d"] or \
        _mismatch(meta["ablations"][name], meta["stages"][2]["digests"]) != []


def test_alph_kdiv_bit_exact_vs_reference():
    meta, a, m, _ = load("tos_seeded_9x7x8")
    p = {k: meta[k] for k in PARAMS}
    ak = meta["alph_kdiv"]
    for stage in ak["stages"]:
        orc.terrain_open_stage(a, m, nrk=stage["nrk"], alph=ak["alph"], kdiv=ak["kdiv"], **p)
        assert _mismatch(digests(a), stage["digests"]) == []


def test_uniform_edge_weights_are_fornberg_quadratic():
    # exactly (1.875, -1.25, 0.375) where the float32 levels are equally
    # spaced; a dz whose half-levels round unevenly moves them by ulps
    for nk, dz in ((5, 200.0), (40, 500.0), (80, 250.0)):
        assert orc.edge_weights(nk, dz) == ((1.875, -1.25, 0.375), (1.875, -1.25, 0.375))
    cgs, cgt = orc.edge_weights(8, 333.3)
    assert cgs == pytest.approx((1.875, -1.25, 0.375), abs=2e-6)
    assert cgt == pytest.approx((1.875, -1.25, 0.375), abs=2e-6)


def _differs(x, y) -> bool:
    return not np.array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32))


def _stretched_column(m, ni, nj, nk, lv):
    from tests.test_oracle_momentum import _padded_rho0

    return {"sigma": lv.sigma, "sigmaf": lv.sigmaf, "rds": lv.rds, "rdsf": lv.rdsf, "ztop": lv.ztop_m,
            "rho0p": _padded_rho0(m["rho0_3d"], ni, nj, nk)}


@pytest.mark.parametrize("ni,nj,nk,dz", [(9, 7, 6, 200.0), (12, 5, 10, 250.0)])
def test_stretched_terrain_stage_on_a_uniform_column_is_the_uniform_stage(ni, nj, nk, dz):
    """The stretched terrain-column restatement (the reference's profile-bound
    acoustic texts, src/cm1core/cuda_gm1_child_psolver3_open.py:152-330) on a
    uniform column with a horizontally uniform base density reproduces the
    twin-pinned uniform stage word for word over three RK stages."""
    from gm1_b200.vertical import uniform_vertical_levels
    from tests.golden.make_golden import terrain_open_fixture

    a, m = terrain_open_fixture(ni, nj, nk, 40 + ni)
    m["rho0_3d"][:] = m["rho0_3d"][:, :1, :1]
    lv = uniform_vertical_levels(nk, dz)
    col = _stretched_column(m, ni, nj, nk, lv)
    p = dict(ni=ni, nj=nj, nk=nk, dt=2.0, nsound=6, dx=450.0, dy=520.0)
    want, got = {k: v.copy() for k, v in a.items()}, {k: v.copy() for k, v in a.items()}
    for nrk in (1, 2, 3):
        orc.terrain_open_stage(want, m, nrk=nrk, dz=dz, **p)
        orc.terrain_open_stage_column(got, m, col, nrk=nrk, **p)
    assert [n for n in orc.ARRAY_NAMES if _differs(got[n], want[n])] == []


def test_stretched_terrain_stage_moves_with_the_profiles():
    """On a stretched column (20 m at the ground to 200 m aloft) and a
    horizontally varying base density the stage differs from the uniform one
    in the prognostic winds and pressure, and stays finite."""
    from gm1_b200.vertical import build_vertical_levels
    from tests.golden.make_golden import terrain_open_fixture

    ni, nj, nk = 9, 8, 10
    a, m = terrain_open_fixture(ni, nj, nk, 77)
    lv = build_vertical_levels(stretch_z=1, nk=nk, dz_m=100.0, ztop_m=1100.0, str_bot_m=40.0, str_top_m=700.0,
                               dz_bot_m=20.0, dz_top_m=200.0)
    col = _stretched_column(m, ni, nj, nk, lv)
    p = dict(ni=ni, nj=nj, nk=nk, nrk=2, dt=2.0, nsound=6, dx=450.0, dy=520.0)
    want, got = {k: v.copy() for k, v in a.items()}, {k: v.copy() for k, v in a.items()}
    orc.terrain_open_stage(want, m, dz=110.0, **p)
    orc.terrain_open_stage_column(got, m, col, **p)
    for n in ("u3d", "v3d", "w3d", "pp3d"):
        assert np.isfinite(got[n]).all() and _differs(got[n], want[n]), n


def _flat_column(nk):
    from gm1_b200.vertical import build_vertical_levels

    spec = {10: (1100.0, 40.0, 700.0), 14: (1630.0, 40.0, 1030.0)}[nk]
    lv = build_vertical_levels(stretch_z=1, nk=nk, dz_m=100.0, ztop_m=spec[0], str_bot_m=spec[1], str_top_m=spec[2],
                               dz_bot_m=20.0, dz_top_m=200.0)
    return {"mh": lv.mh, "mf": lv.mf, "rdz": float(np.float32(1.0) / np.float32(100.0))}


def test_flat_stage_keeps_a_resting_atmosphere_at_rest():
    """The flat-column restatement (sound.F's terrain_flag=.false. texts,
    src/cm1core/cuda_gm1_child_psolver3_open.py:343-507, in the order of
    :1618-1795) leaves a state with no wind, no perturbation pressure and no
    tendencies unchanged, on every lateral family it takes."""
    from tests.golden.make_golden import terrain_open_fixture

    ni, nj, nk = 9, 8, 10
    a, m = terrain_open_fixture(ni, nj, nk, 11)
    for n in ("u3d", "ua", "uten", "v3d", "va", "vten", "w3d", "wa", "wten", "ppi", "pp3d", "ppx", "ppten"):
        a[n][:] = 0.0
    for obc in (0x2222, 0x2211, 0x1111):
        got = {k: v.copy() for k, v in a.items()}
        for nrk in (1, 2, 3):
            orc.terrain_open_stage_flat(got, m, _flat_column(nk), ni=ni, nj=nj, nk=nk, nrk=nrk, dt=2.0, nsound=6,
                                        dx=450.0, dy=520.0, obc=obc)
        for n in ("u3d", "v3d", "w3d", "pp3d", "ppd"):
            assert not np.any(got[n][1:nk + 1]), (hex(obc), n)


def test_flat_stage_lateral_family_moves_the_boundary_faces():
    """Periodic and open west/east sides take different boundary-face
    updates (the pressure gradient's dtu0 mask against the open-side
    radiation update); the stage stays finite on both."""
    from tests.golden.make_golden import terrain_open_fixture

    ni, nj, nk = 12, 9, 10
    a, m = terrain_open_fixture(ni, nj, nk, 12)
    p = dict(ni=ni, nj=nj, nk=nk, nrk=1, dt=2.0, nsound=6, dx=450.0, dy=520.0)
    only = orc.ablation_mask(between_step_pressure_fill=False, radiation_history_production=False,
                             stage_family_fills=False)
    one, two = {k: v.copy() for k, v in a.items()}, {k: v.copy() for k, v in a.items()}
    orc.terrain_open_stage_flat(one, m, _flat_column(nk), obc=0x2222, ablations=only, **p)
    orc.terrain_open_stage_flat(two, m, _flat_column(nk), obc=0x2211, ablations=only, **p)
    # u faces x = 3 and x = ni+3 are the west and east boundary faces
    assert _differs(one["u3d"][1:nk + 1, 3:nj + 3, 3], two["u3d"][1:nk + 1, 3:nj + 3, 3])
    assert np.isfinite(one["pp3d"]).all() and np.isfinite(two["pp3d"]).all()
