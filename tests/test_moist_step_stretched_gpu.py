"""The composed moist large step on a stretched column (the flat,
terrain_flag=.false., operator family of the reference's Cartesian
stretched lane: flat calcdef/turbt/TKE advection, stretched-column scalar
advection, pdef chain, momentum, post-acoustic flux, flat buoyancy and the
flat acoustic stage) on the GPU against the same composition of the oracle's
operators, after 1, 3 and 60 large steps, including the 80-level supercell
column of the 640x768x80 configuration on a reduced plane.

Bars (tests/moist_common.py measures each field on its own scale):
SHORT_BARS after 1 and 3 steps; over 60 steps, the GPU's worst error against
the FP64 run of the same operators at most sixteen times the binary32
oracle's own (tests/fp64_common.py: LONG_RUN_FACTOR).  The words differ
only where Kessler and the TKE closure pass values through powf, expf and
sqrtf (CUDA and the C library round their last bits differently) and the
rest of the step carries those ulps."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.moist_step import (SUPERCELL_STRETCHED_COLUMN, MoistLargeStep, MoistStepConfig, StretchedColumnSpec,
                                 upload, weisman_klemp_initial_state)
from oracle.moist_composition import OracleMoistStep
from tests.fp64_common import check_long_run
from tests.moist_common import SHORT_BARS, check_errors, field_errors, format_errors

pytestmark = pytest.mark.gpu

SHALLOW = StretchedColumnSpec(1630.0, 40.0, 1030.0, 20.0, 200.0)  # nk = 14: 20 m at the ground, 1.63 km lid
STRETCHED_BARS = SHORT_BARS


def _pair(ni, nj, nk, column, seed=7, with_host=False, **kw):
    cfg = MoistStepConfig(ni, nj, nk, 100.0, 100.0, 100.0, 0.6, 8, column=column)
    init = dict(seed=seed, bubble_radius_m=(800.0, 400.0), bubble_center_z_m=400.0, bubble_cloud=1.0e-3,
                bubble_rain=5.0e-4)
    init.update(kw)
    host, metrics = weisman_klemp_initial_state(cfg, **init)
    dev = MoistLargeStep(cfg, upload(host), upload(metrics))
    ref = OracleMoistStep(cfg, {k: v.copy() for k, v in host.items()}, {k: v.copy() for k, v in metrics.items()})
    if with_host:
        return cfg, dev, ref, host, metrics
    return cfg, dev, ref


@pytest.mark.parametrize("grid", [(24, 20), (70, 40)])
def test_stretched_step_matches_oracle_composition(grid):
    _, dev, ref = _pair(*grid, 14, SHALLOW)
    for step in (1, 2, 3):
        dev.step()
        ref.step()
        torch.cuda.synchronize()
        if step in (1, 3):
            err = field_errors(dev.s, ref.s)
            print(grid, "after", step, format_errors(err))
            check_errors(err, STRETCHED_BARS, f"{grid} step {step}")
    assert float(ref.s["q3d"][2].max()) > 0.0 and float(ref.s["rain"].max()) > 0.0
    dev.check()


def test_supercell_column_on_a_reduced_plane():
    """The 80-level column of the 640x768x80 configuration (20 m at the
    ground to 500 m aloft, lid 20.8 km) on a 48x40 plane, 3 steps."""
    _, dev, ref = _pair(48, 40, 80, SUPERCELL_STRETCHED_COLUMN, seed=2, bubble_radius_m=(1500.0, 1400.0),
                        bubble_center_z_m=1500.0)
    for step in (1, 2, 3):
        dev.step()
        ref.step()
        torch.cuda.synchronize()
        if step in (1, 3):
            err = field_errors(dev.s, ref.s)
            print("supercell column after", step, format_errors(err))
            check_errors(err, STRETCHED_BARS, f"supercell column step {step}")
    dev.check()


@pytest.mark.parametrize("case", ["shallow", "supercell"])
def test_stretched_step_stays_bounded_over_60_steps(case):
    if case == "shallow":
        cfg, dev, ref, host, metrics = _pair(32, 28, 14, SHALLOW, seed=11, with_host=True)
    else:
        cfg, dev, ref, host, metrics = _pair(32, 32, 80, SUPERCELL_STRETCHED_COLUMN, seed=13, with_host=True,
                                             bubble_radius_m=(1200.0, 1400.0), bubble_center_z_m=1500.0)
    del dev, ref
    check_long_run(cfg, host, metrics, lambda c, h, m: MoistLargeStep(c, upload(h), upload(m)), what=case)


def test_stretched_graph_replay_and_concurrency_give_the_sequential_words():
    cfg = MoistStepConfig(40, 33, 14, 100.0, 100.0, 100.0, 0.6, 8, column=SHALLOW)
    host, metrics = weisman_klemp_initial_state(cfg, seed=5, bubble_radius_m=(800.0, 400.0), bubble_center_z_m=400.0,
                                                bubble_cloud=1.0e-3, bubble_rain=5.0e-4)
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
    for n in ("u3d", "v3d", "w3d", "th3d", "pp3d", "q3d", "tke3d", "rain", "ppx", "tha", "qa"):
        assert np.array_equal(seq.s[n].cpu().numpy().view(np.uint32), con.s[n].cpu().numpy().view(np.uint32)), n
