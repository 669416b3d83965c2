"""The whole moist step through the C ABI (gm1b_moist_large_step, driven by
ctypes alone through NativeMoistLargeStep) against the Python composition
MoistLargeStep: the same launches in the same order, so every word of every
state array the step writes must be identical, on the uniform and on the
stretched column, sequential and concurrent, eager and captured in a CUDA
graph; and the folded failure words read back through the ABI."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.moist_step import (CourantStop, MoistLargeStep, MoistStepConfig, NativeMoistLargeStep,
                                 StretchedColumnSpec, upload, weisman_klemp_initial_state)

pytestmark = pytest.mark.gpu

SHALLOW = StretchedColumnSpec(1630.0, 40.0, 1030.0, 20.0, 200.0)
COMPARED = ("ua", "u3d", "va", "v3d", "wa", "w3d", "ppi", "pp3d", "ppx", "tha", "th3d", "qa", "q3d", "tkea", "tke3d",
            "rho", "rr", "rf", "prs", "rain", "prate", "asq", "qbudget", "qpten", "qtten", "qvten", "qcten", "kmh",
            "kmv", "divx", "rru", "rrv", "rrw", "radbcw", "radbce", "radbcs", "radbcn")


def _case(stretched: bool):
    if stretched:
        cfg = MoistStepConfig(40, 33, 14, 100.0, 100.0, 100.0, 0.6, 8, column=SHALLOW)
        init = dict(seed=5, bubble_radius_m=(800.0, 400.0), bubble_center_z_m=400.0)
    else:
        cfg = MoistStepConfig(40, 33, 16, 1000.0, 1000.0, 250.0, 5.0, 10)
        init = dict(seed=5, bubble_radius_m=(6000.0, 1400.0))
    host, metrics = weisman_klemp_initial_state(cfg, bubble_cloud=1.0e-3, bubble_rain=5.0e-4, **init)
    return cfg, host, metrics


def _same(a, b, names=COMPARED):
    bad = []
    for n in names:
        x, y = a[n].cpu().numpy(), b[n].cpu().numpy()
        if not np.array_equal(x.view(np.uint8), y.view(np.uint8)):
            bad.append(n)
    return bad


@pytest.mark.parametrize("stretched", [False, True])
@pytest.mark.parametrize("concurrent", [False, True])
def test_native_step_gives_the_python_composition_words(stretched, concurrent):
    cfg, host, metrics = _case(stretched)
    py = MoistLargeStep(cfg, upload(host), upload(metrics), concurrent=False)
    nat = NativeMoistLargeStep(cfg, upload(host), upload(metrics), concurrent=concurrent)
    for _ in range(2):
        py.step()
        nat.step()
    torch.cuda.synchronize()
    assert _same(py.s, nat.s) == []
    st_py, st_nat = py.check(current_state=False), nat.check()
    assert st_nat["courant_samples"] == 2 and st_nat["kessler_samples"] == 2
    assert st_nat["max_courant"] == st_py["max_courant"]
    assert st_nat["max_fall_substeps"] == st_py["max_fall_substeps"]
    nat.close()


def test_native_step_replays_from_a_cuda_graph():
    cfg, host, metrics = _case(True)
    eager = NativeMoistLargeStep(cfg, upload(host), upload(metrics))
    stream = torch.cuda.Stream()
    graphed = NativeMoistLargeStep(cfg, upload(host), upload(metrics), stream=stream)
    eager.step()
    eager.step()
    with torch.cuda.stream(stream):
        graphed.step()  # the first step outside the capture configures the kernels
    stream.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        graphed.step()
    graph.replay()
    torch.cuda.synchronize()
    assert _same(eager.s, graphed.s) == []
    del graph
    eager.close()
    graphed.close()


def test_native_step_refuses_a_courant_stop():
    cfg, host, metrics = _case(False)
    host["u3d"][3:8, 8:10, 10:12] = np.float32(400.0)
    host["ua"][:] = host["u3d"]
    nat = NativeMoistLargeStep(cfg, upload(host), upload(metrics))
    nat.step()
    rc, words = nat.status()
    assert rc == 2 and words["max_courant"] >= 1.5
    with pytest.raises(CourantStop):
        nat.check()
    nat.close()
