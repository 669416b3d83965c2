"""Parity of the CUDA periodic lane, called through the C ABI, with the
reference (golden vectors made by the reference's own CPU twins) and with the
CPU oracle at full size.  Bar: every float32 word bit-identical
(max_ulp 0, the reference's raw-bit comparer semantics,
src/cm1core/cuda_psolver3_trajectory.py:904-938)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.arrays import ALL_ARRAY_NAMES, SCRATCH_OUTPUT_NAMES, SOUND_ARRAY_NAMES, TRAJECTORY_STATE_NAMES
from gm1_b200.initial_state import DRY_BUBBLE_64, dry_periodic_state
from gm1_b200.periodic import (
    BarrierTimeout,
    TrajectoryAblations,
    launch_cuda_psolver3_trajectory,
    launch_cuda_sound3_periodic_three_stage,
    to_device,
    to_host,
)
from oracle import periodic as orc
from tests._golden import bit_mismatches, digest, load_json, load_npz

pytestmark = pytest.mark.gpu


def _run_sound(inputs, meta, scratch=True):
    dev = to_device(inputs)
    keys = ("ni", "nj", "nk", "dt", "nsound", "rdx", "rdy", "rdz")
    launch = launch_cuda_sound3_periodic_three_stage(dev, scratch_outputs=scratch, **{k: meta[k] for k in keys})
    launch.ready_event.synchronize()
    return to_host(dev), launch


@pytest.mark.parametrize("tag", ["sound3_5x4x7", "sound3_8x6x12"])
def test_sound3_three_stage_bit_exact_vs_reference(tag):
    meta, inputs, expected = load_npz(tag)
    got, launch = _run_sound(inputs, meta)
    assert [c["nloop"] for c in launch.receipt["cadence"]] == meta["nloop"]
    assert bit_mismatches(expected, got, SOUND_ARRAY_NAMES) == {}


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("tag", ["sound3_5x4x7", "sound3_8x6x12"])
def test_sound3_without_scratch_outputs_keeps_state_bits(tag, fused):
    """Both stage paths without scratch outputs: the persistent one-kernel
    stage (fused) and two launches per small step."""
    meta, inputs, expected = load_npz(tag)
    dev = to_device(inputs)
    keys = ("ni", "nj", "nk", "dt", "nsound", "rdx", "rdy", "rdz")
    launch = launch_cuda_sound3_periodic_three_stage(dev, scratch_outputs=False, fused_stage=fused,
                                                     **{k: meta[k] for k in keys})
    launch.ready_event.synchronize()
    got = to_host(dev)
    state = ("u3d", "v3d", "w3d", "pp3d", "ppx", "ppd", "rru", "rrv", "rrw", "qk", "pk1", "pk2", "mm")
    assert bit_mismatches(expected, got, state) == {}
    if fused:  # barrier status word of the fused stage: no barrier gave up
        assert int(got["tri_residual"].reshape(-1)[:3].view(np.int32)[2]) == 0


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("tag", ["traj_7x6x7", "traj_9x5x8"])
def test_trajectory_fast_paths_match_reference_on_state_words(tag, fused):
    """The benchmark path on the reference's golden trajectories: every array
    except the acoustic scratch outputs bit-identical."""
    meta, inputs, expected = load_npz(tag)
    dev = to_device(inputs)
    keys = ("ni", "nj", "nk", "steps", "dt", "nsound", "dx", "dy", "dz")
    launch = launch_cuda_psolver3_trajectory(dev, scratch_outputs=False, fused_stage=fused,
                                             **{k: meta[k] for k in keys})
    launch.ready_event.synchronize()
    got = to_host(dev)
    names = [n for n in ALL_ARRAY_NAMES if n not in SCRATCH_OUTPUT_NAMES]
    assert bit_mismatches(expected, got, names) == {}


@pytest.mark.parametrize("tag", ["traj_7x6x7", "traj_9x5x8"])
def test_trajectory_bit_exact_vs_reference(tag):
    meta, inputs, expected = load_npz(tag)
    dev = to_device(inputs)
    keys = ("ni", "nj", "nk", "steps", "dt", "nsound", "dx", "dy", "dz")
    launch = launch_cuda_psolver3_trajectory(dev, **{k: meta[k] for k in keys})
    launch.ready_event.synchronize()
    got = to_host(dev)
    assert bit_mismatches(expected, got, ALL_ARRAY_NAMES) == {}


def test_trajectory_ablations_match_reference_digests():
    from tests.golden.make_golden import SMALL_CASE  # noqa: PLC0415

    case = SMALL_CASE
    record = load_json("traj_ablations_7x6x7.json")
    p = dict(ni=case.ni, nj=case.nj, nk=case.nk, steps=1, dt=case.dt, nsound=case.nsound,
             dx=case.dx, dy=case.dy, dz=case.dz)
    for field, entry in record.items():
        dev = to_device(dry_periodic_state(case))
        launch_cuda_psolver3_trajectory(dev, ablations=TrajectoryAblations(**{field: False}), **p)
        torch.cuda.synchronize()
        got = to_host(dev)
        bad = [n for n in ALL_ARRAY_NAMES if digest(got[n]) != entry["digests"][n]]
        assert bad == [], (field, bad)


def _c1_params(steps):
    c = DRY_BUBBLE_64
    return dict(ni=c.ni, nj=c.nj, nk=c.nk, steps=steps, dt=c.dt, nsound=c.nsound, dx=c.dx, dy=c.dy, dz=c.dz)


def test_c1_full_size_matches_oracle_after_1_and_10_steps():
    host = dry_periodic_state(DRY_BUBBLE_64)
    dev = to_device(host)
    # 1 step
    launch_cuda_psolver3_trajectory(dev, **_c1_params(1))
    orc.traj_steps(host, **_c1_params(1))
    torch.cuda.synchronize()
    assert bit_mismatches(host, to_host(dev), ALL_ARRAY_NAMES) == {}
    # 9 more
    launch_cuda_psolver3_trajectory(dev, **_c1_params(9))
    orc.traj_steps(host, **_c1_params(9))
    torch.cuda.synchronize()
    got = to_host(dev)
    assert bit_mismatches(host, got, ALL_ARRAY_NAMES) == {}
    # size-independent properties of the state after 10 steps
    nk, nj, ni = DRY_BUBBLE_64.nk, DRY_BUBBLE_64.nj, DRY_BUBBLE_64.ni
    assert not np.any(got["w3d"][1].view(np.uint32)) and not np.any(got["w3d"][nk + 1].view(np.uint32))
    assert np.all(np.isfinite(got["th3d"])) and float(np.max(np.abs(got["w3d"]))) > 0.0
    res = got["tri_residual"][2 : nk + 1, 1 : nj + 1, 1 : ni + 1]
    assert float(np.max(np.abs(res))) < 2.0e-6


def test_c1_matches_reference_digests():
    from tests._golden import GOLDEN  # noqa: PLC0415

    if not (GOLDEN / "traj_c1_digests.json").exists():
        pytest.skip("full-size reference digests not generated yet")
    record = load_json("traj_c1_digests.json")
    host = dry_periodic_state(DRY_BUBBLE_64)
    assert {n: digest(host[n]) for n in ALL_ARRAY_NAMES} == record["input_digests"]
    dev = to_device(host)
    done = 0
    for step in sorted(int(s) for s in record["steps"]):
        launch_cuda_psolver3_trajectory(dev, **_c1_params(step - done))
        done = step
        torch.cuda.synchronize()
        got = to_host(dev)
        want = record["steps"][str(step)]["digests"]
        bad = [n for n in ALL_ARRAY_NAMES if digest(got[n]) != want[n]]
        assert bad == [], (step, bad)


@pytest.mark.parametrize("fused", [True, False])
def test_fast_path_without_scratch_outputs_keeps_every_state_word(fused):
    """The benchmark path (no scratch outputs: stage-constant tridiagonal
    coefficients reused across small steps; with ``fused`` each acoustic
    stage is one persistent kernel) is bit-identical to the oracle on every
    array except the acoustic scratch it repurposes."""
    host = dry_periodic_state(DRY_BUBBLE_64)
    dev = to_device(host)
    launch_cuda_psolver3_trajectory(dev, scratch_outputs=False, fused_stage=fused, **_c1_params(3))
    orc.traj_steps(host, **_c1_params(3))
    torch.cuda.synchronize()
    got = to_host(dev)
    names = [n for n in TRAJECTORY_STATE_NAMES if n not in ("tri_pivot", "tri_residual")]
    assert bit_mismatches(host, got, names) == {}
    names = [n for n in ALL_ARRAY_NAMES if n not in SCRATCH_OUTPUT_NAMES]
    assert bit_mismatches(host, got, names) == {}
    if fused:
        words = got["tri_residual"].reshape(-1)[:3].view(np.int32)
        assert int(words[2]) == 0
        # 64-bit arrive count after the last stage: (nloop - 1) barriers x 128 CTAs
        count = int(got["tri_residual"].reshape(-1)[:2].view(np.uint64)[0])
        assert count == 5 * 2 * 64


def test_repeat_runs_are_bit_identical_and_streams_are_honoured():
    host = dry_periodic_state(DRY_BUBBLE_64)
    one = to_device(host)
    two = to_device(host)
    s = torch.cuda.Stream()
    launch_cuda_psolver3_trajectory(one, **_c1_params(2))
    with torch.cuda.stream(s):
        launch = launch_cuda_psolver3_trajectory(two, stream=s, **_c1_params(2))
    launch.ready_event.synchronize()
    torch.cuda.synchronize()
    for n in TRAJECTORY_STATE_NAMES:
        assert torch.equal(one[n].view(torch.int32), two[n].view(torch.int32)), n


def test_launch_rejects_bad_device_arrays():
    host = dry_periodic_state(DRY_BUBBLE_64)
    dev = to_device(host)
    bad = dict(dev)
    bad["u3d"] = dev["u3d"].double()
    with pytest.raises(ValueError, match="invalid CUDA dtype"):
        launch_cuda_psolver3_trajectory(bad, **_c1_params(1))
    bad = dict(dev)
    bad["va"] = dev["ua"]
    with pytest.raises(ValueError):
        launch_cuda_psolver3_trajectory(bad, **_c1_params(1))
    bad = dict(dev)
    bad["tha"] = dev["th3d"]
    with pytest.raises(ValueError, match="alias"):
        launch_cuda_psolver3_trajectory(bad, **_c1_params(1))


def test_persistent_stage_barrier_timeout_is_reported_and_context_survives():
    """The persistent acoustic stage's grid barrier waits at most
    barrier_spin_limit polls.  With a limit of one poll the CTAs that reach a
    barrier first give up before the rest arrive: the kernel returns, the
    status word reports it and the launcher raises.  The context stays
    usable: the same trajectory with the default limit afterwards matches the
    oracle word for word."""
    p = _c1_params(1)
    dev = to_device(dry_periodic_state(DRY_BUBBLE_64))
    with pytest.raises(BarrierTimeout):
        launch_cuda_psolver3_trajectory(dev, scratch_outputs=False, barrier_spin_limit=1, **p)
    host = dry_periodic_state(DRY_BUBBLE_64)
    dev = to_device(host)
    launch = launch_cuda_psolver3_trajectory(dev, scratch_outputs=False, **p)
    assert int(launch.barrier_status.item()) == 0
    orc.traj_steps(host, **p)
    got = to_host(dev)
    names = [n for n in ALL_ARRAY_NAMES if n not in SCRATCH_OUTPUT_NAMES]
    assert bit_mismatches(host, got, names) == {}
