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
