"""Pins the CPU oracle to golden vectors produced by the reference itself.

The fixtures hold whole input/output array sets of the reference's NumPy twins
(cpu_sound3_periodic_three_stage_inplace, cpu_psolver3_trajectory_inplace) and
digests of its ablation runs; the oracle must reproduce every word.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests._golden import bit_mismatches, digest, load_json, load_npz
from gm1_b200.arrays import ALL_ARRAY_NAMES, SOUND_ARRAY_NAMES
from gm1_b200.initial_state import DryBubbleCase, dry_periodic_state
from oracle import periodic as orc


@pytest.mark.parametrize("tag", ["sound3_5x4x7", "sound3_8x6x12"])
def test_oracle_sound3_three_stage_matches_reference_bits(tag):
    meta, inputs, expected = load_npz(tag)
    keys = ("ni", "nj", "nk", "dt", "nsound", "rdx", "rdy", "rdz")
    nloops = orc.sound3_periodic_three_stage(inputs, **{k: meta[k] for k in keys})
    assert nloops == meta["nloop"]
    assert bit_mismatches(expected, inputs, SOUND_ARRAY_NAMES) == {}


@pytest.mark.parametrize("tag", ["traj_7x6x7", "traj_9x5x8"])
def test_oracle_trajectory_matches_reference_bits(tag):
    meta, inputs, expected = load_npz(tag)
    keys = ("ni", "nj", "nk", "steps", "dt", "nsound", "dx", "dy", "dz")
    orc.traj_steps(inputs, **{k: meta[k] for k in keys})
    assert bit_mismatches(expected, inputs, ALL_ARRAY_NAMES) == {}


def test_oracle_stagewise_cadence_matches_reference():
    meta, inputs, _ = load_npz("traj_7x6x7")
    ni, nj, nk = meta["ni"], meta["nj"], meta["nk"]
    p = dict(ni=ni, nj=nj, nk=nk, dt=meta["dt"], nsound=meta["nsound"], dx=meta["dx"], dy=meta["dy"], dz=meta["dz"])
    got = []
    for _step in range(meta["steps"]):
        for nrk in (1, 2, 3):
            nloop = orc.traj_stage(inputs, nrk=nrk, **p)
            res = inputs["tri_residual"][2 : nk + 1, 1 : nj + 1, 1 : ni + 1]
            got.append((nrk, nloop, float(np.max(np.abs(res), initial=np.float32(0)))))
        orc.traj_post_step(inputs, ni=ni, nj=nj, nk=nk)
    want = [(c["nrk"], c["nloop"], c["max_tridiagonal_residual"]) for c in meta["cadence"]]
    assert got == want
    assert [(c["nrk"], c["nloop"]) for c in meta["cadence"][:3]] == [(1, 2), (2, 3), (3, 6)]


def test_oracle_ablations_match_reference_digests():
    from tests.golden.make_golden import SMALL_CASE  # noqa: PLC0415

    record = load_json("traj_ablations_7x6x7.json")
    case = SMALL_CASE
    p = dict(ni=case.ni, nj=case.nj, nk=case.nk, steps=1, dt=case.dt, nsound=case.nsound,
             dx=case.dx, dy=case.dy, dz=case.dz)
    seen = set()
    for field, entry in record.items():
        a = dry_periodic_state(case)
        orc.traj_steps(a, ablations=entry["mask"], **p)
        got = {n: digest(a[n]) for n in ALL_ARRAY_NAMES}
        assert got == entry["digests"], field
        seen.add(tuple(sorted(got.items())))
    # every ablation changes the result (reference test_cuda_psolver3_trajectory.py:197-215)
    assert len(seen) == len(record)


def test_oracle_schedule_matches_reference_table():
    for dt, nsound, nrk, nloop, dts in load_json("schedule.json"):
        assert orc.stage_schedule(dt, nsound, nrk) == (nloop, dts)
