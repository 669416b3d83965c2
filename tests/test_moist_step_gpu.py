"""The composed moist large step on the GPU against the same composition of
the oracle's operators, on Weisman-Klemp starts with cloud and rain in the
bubble (so every Kessler branch runs from the first step), after 1 and
after 3 large steps, on a small and on a multi-tile grid.

Stated tolerance (Kessler and the TKE closure pass values through powf,
expf and sqrtf, whose last bits differ between CUDA and the C library, and
the acoustic, advection and pdef arithmetic then carries those ulps): each
prognostic field measured on its own scale (the largest |value| of that
field: u, v, w each, theta', pi', qv, qc, qr each, TKE) within
tests/moist_common.py's SHORT_BARS after 1 and 3 steps (also at the full
256x256x80 size after one step); over 60 steps, the GPU's worst error
against the FP64 run of the same operators at most sixteen times the binary32
oracle's own (tests/fp64_common.py: LONG_RUN_FACTOR); u, v and w are word-identical after
one step.  A CUDA-graph replay of the step gives the
eager words."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.moist_step import (CourantStop, MoistLargeStep, MoistStepConfig, SatadjNonConvergence, upload,
                                 weisman_klemp_initial_state)
from oracle.moist_composition import OracleMoistStep
from tests.fp64_common import check_long_run
from tests.moist_common import SHORT_BARS, check_errors, field_errors, format_errors

pytestmark = pytest.mark.gpu

# each field on its own scale (tests/moist_common.py): SHORT_BARS after 1
# and 3 steps; over 60 steps, the FP64 run (tests/fp64_common.py)
OWN_BARS = SHORT_BARS

FIELDS = ("u3d", "v3d", "w3d", "th3d", "pp3d", "q3d", "tke3d")
MAX_REL, RMS_REL = 1.0e-4, 1.0e-5


def _scale(name, s):
    if name == "th3d":
        return float(np.max(np.abs(s["th0_3d"].astype(np.float64) + s["th3d"])))
    if name == "pp3d":
        return float(np.max(np.abs(s["pi0"]))) + float(np.max(np.abs(s["pp3d"])))
    if name == "q3d":
        return float(np.max(s["q3d"][:3].sum(axis=0)))
    if name in ("u3d", "v3d", "w3d"):
        return max(float(np.max(np.abs(s[n]))) for n in ("u3d", "v3d", "w3d"))
    return float(np.max(np.abs(s[name])))


def _errors(gpu, ref):
    out = {}
    for n in FIELDS:
        g, r = gpu[n].cpu().numpy().astype(np.float64), ref[n].astype(np.float64)
        d = g - r
        sc = _scale(n, ref)
        out[n] = (float(np.max(np.abs(d))) / sc, float(np.sqrt(np.mean(d * d))) / sc)
    return out


@pytest.mark.parametrize("grid", [(24, 20, 16), (70, 40, 20)])
def test_composed_step_matches_oracle_composition(grid):
    ni, nj, nk = grid
    cfg = MoistStepConfig(ni, nj, nk, 1000.0, 1000.0, 250.0, 5.0, 10)
    host, metrics = weisman_klemp_initial_state(cfg, seed=7, bubble_radius_m=(6000.0, 1400.0),
                                                bubble_cloud=1.0e-3, bubble_rain=5.0e-4)
    dev = MoistLargeStep(cfg, upload(host), upload(metrics))
    ref = OracleMoistStep(cfg, {k: v.copy() for k, v in host.items()}, {k: v.copy() for k, v in metrics.items()})
    for step in (1, 2, 3):
        dev.step()
        ref.step()
        torch.cuda.synchronize()
        if step in (1, 3):
            err = _errors(dev.s, ref.s)
            print(grid, "after", step, {n: (f"{a:.2e}", f"{b:.2e}") for n, (a, b) in err.items()})
            for n, (mx, rms) in err.items():
                assert mx <= MAX_REL and rms <= RMS_REL, (n, step, mx, rms)
            own = field_errors(dev.s, ref.s)
            print(grid, "after", step, "own scale:", format_errors(own))
            check_errors(own, OWN_BARS, f"{grid} step {step}")
    assert float(ref.s["q3d"][2].max()) > 0.0 and float(ref.s["rain"].max()) > 0.0


def test_composed_step_stays_bounded_over_60_steps():
    ni, nj, nk = 32, 28, 16
    cfg = MoistStepConfig(ni, nj, nk, 1000.0, 1000.0, 250.0, 5.0, 10)
    host, metrics = weisman_klemp_initial_state(cfg, seed=11, bubble_radius_m=(6000.0, 1400.0),
                                                bubble_cloud=1.0e-3, bubble_rain=5.0e-4)
    check_long_run(cfg, host, metrics, lambda c, h, m: MoistLargeStep(c, upload(h), upload(m)), what="uniform")


def test_full_size_256x256x80_step_matches_oracle_composition():
    """One step of the 256x256x80 Weisman-Klemp workload itself (the
    benchmark's configuration 2) against the oracle composition run on all
    host cores."""
    from oracle import periodic as orc

    orc.set_threads(orc.max_threads())
    cfg = MoistStepConfig(256, 256, 80, 1000.0, 1000.0, 250.0, 5.0, 10)
    host, metrics = weisman_klemp_initial_state(cfg, seed=2, bubble_radius_m=(10000.0, 1500.0),
                                                bubble_center_z_m=1500.0)
    dev = MoistLargeStep(cfg, upload(host), upload(metrics))
    ref = OracleMoistStep(cfg, host, metrics)
    dev.step()
    ref.step()
    torch.cuda.synchronize()
    err = field_errors(dev.s, ref.s)
    print("256x256x80 after 1 step:", format_errors(err))
    check_errors(err, OWN_BARS, "256x256x80 step 1")
    dev.check()


def test_graph_replay_gives_the_eager_words():
    ni, nj, nk = 40, 33, 16
    cfg = MoistStepConfig(ni, nj, nk, 1000.0, 1000.0, 250.0, 5.0, 10)
    host, metrics = weisman_klemp_initial_state(cfg, seed=3, bubble_cloud=1.0e-3, bubble_rain=5.0e-4)
    eager = MoistLargeStep(cfg, upload(host), upload(metrics))
    stream = torch.cuda.Stream()
    graphed = MoistLargeStep(cfg, upload(host), upload(metrics), stream=stream)
    eager.step()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        graphed.step()
    graph.replay()
    torch.cuda.synchronize()
    for n in FIELDS:
        assert torch.equal(eager.s[n].view(torch.int32), graphed.s[n].view(torch.int32)), n


def test_concurrent_stage_tail_gives_the_sequential_words():
    """The concurrent step (scalars, boundaries and TKE of each stage on side
    streams) writes the same words as the same step run operation by
    operation on one stream, including when captured as a CUDA graph."""
    ni, nj, nk = 40, 33, 16
    cfg = MoistStepConfig(ni, nj, nk, 1000.0, 1000.0, 250.0, 5.0, 10)
    host, metrics = weisman_klemp_initial_state(cfg, seed=5, bubble_cloud=1.0e-3, bubble_rain=5.0e-4)
    seq = MoistLargeStep(cfg, upload(host), upload(metrics), concurrent=False)
    stream = torch.cuda.Stream()
    con = MoistLargeStep(cfg, upload(host), upload(metrics), stream=stream, concurrent=True)
    for _ in range(2):
        seq.step()
    with torch.cuda.stream(stream):
        con.step()
    stream.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        con.step()
    graph.replay()
    torch.cuda.synchronize()
    for n in FIELDS + ("rain", "ppx", "tha", "qa"):
        assert np.array_equal(seq.s[n].cpu().numpy().view(np.uint32), con.s[n].cpu().numpy().view(np.uint32)), n


def _cloudy(ni=24, nj=20, nk=16, seed=7):
    cfg = MoistStepConfig(ni, nj, nk, 1000.0, 1000.0, 250.0, 5.0, 10)
    host, metrics = weisman_klemp_initial_state(cfg, seed=seed, bubble_radius_m=(6000.0, 1400.0),
                                                bubble_cloud=1.0e-3, bubble_rain=5.0e-4)
    return cfg, host, metrics


def test_status_words_of_clean_steps():
    """Two ordinary steps: no failure word set, the Courant number of the
    state entering each step and of the current state folded (three
    samples) and finite below CM1's stop, the Kessler words of both steps."""
    cfg, host, metrics = _cloudy()
    dev = MoistLargeStep(cfg, upload(host), upload(metrics))
    dev.step()
    dev.step()
    out = dev.check()
    assert out["satadj_nonconverged_cells"] == 0 and out["blown_up_fall_columns"] == 0
    assert out["courant_samples"] == 3 and out["kessler_samples"] == 2
    assert 0.0 < out["max_courant"] < 1.5 and out["max_fall_substeps"] >= 1


def test_satadj_nonconvergence_is_refused():
    """The step's refusal of a saturation adjustment that ran out of
    iterations: the Kessler operator is run into the step's own workspace
    on a state with a non-converging cell (tests/test_kessler_gpu.py), its
    status words are folded as the step folds them after its Kessler
    transition, and check() refuses as CM1 stops the run.  (Within a step
    the transition recomputes the density from the state's own pressure,
    and no finite state found so far defeats the iteration there.)"""
    from gm1_b200.kessler import Gm1KesslerDriverSelection, launch_cuda_gm1_kessler_driver
    from tests.test_kessler_gpu import nonconvergent_fixture

    cfg, host, metrics = _cloudy()
    dev = MoistLargeStep(cfg, upload(host), upload(metrics))
    a, _ = nonconvergent_fixture(cfg.ni, cfg.nj, cfg.nk)
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in a.items()}
    launch_cuda_gm1_kessler_driver(d, ni=cfg.ni, nj=cfg.nj, nk=cfg.nk, dx=1000.0, dy=1000.0, dz=100.0, dt=5.0,
                                   selection=Gm1KesslerDriverSelection(equation_set=2),
                                   workspace=dev.kessler.workspace)
    dev.fold_kessler_status()
    assert dev.status()["satadj_nonconverged_cells"] >= 1
    with pytest.raises(SatadjNonConvergence):
        dev.check(current_state=False)


def test_courant_stop_is_refused():
    """A 400 m/s jet in a few columns gives an advective Courant number of
    2 at dt = 5 s, dx = 1 km: check() refuses before any step runs."""
    cfg, host, metrics = _cloudy()
    host["u3d"][3:8, 8:10, 10:12] = np.float32(400.0)
    dev = MoistLargeStep(cfg, upload(host), upload(metrics))
    with pytest.raises(CourantStop):
        dev.check()
    assert dev.status()["max_courant"] >= 1.5


def test_tuned_step_gives_the_untuned_words():
    """A step whose scalar-advection z-chunks the autotuner picked for its
    grid leaves the words of the default chunks (the chunk decides which CTA
    forms a level, not the level's words)."""
    from gm1_b200.autotune import Autotuner  # noqa: PLC0415

    cfg = MoistStepConfig(40, 24, 18, 1000.0, 1000.0, 250.0, 5.0, 10)
    host, metrics = weisman_klemp_initial_state(cfg, seed=9, bubble_radius_m=(6000.0, 1400.0), bubble_cloud=1.0e-3)
    tuner = Autotuner()
    tuned = MoistLargeStep(cfg, upload(host), upload(metrics), tuner=tuner)
    plain = MoistLargeStep(cfg, upload(host), upload(metrics))
    assert len(tuner.table) == 2 and all(v["best"] in (1, 2, 4, 8, 16) for v in tuner.table.values())
    for _ in range(2):
        tuned.step()
        plain.step()
    torch.cuda.synchronize()
    for n in FIELDS:
        assert torch.equal(tuned.s[n], plain.s[n]), n
