"""Restart of the composed moist step on the GPU: a run written to a CM1FCP1
envelope after 3 large steps and continued for 3 more from the file, by a
step built afresh from the same configuration and initial state, leaves the
words of 6 uninterrupted steps in every array of the state (the Python
composition on the uniform column, and the C ABI's whole-step entry on the
80-level stretched column); a resume on another configuration or over a
changed base state is refused."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.moist_step import (SUPERCELL_STRETCHED_COLUMN, MoistLargeStep, MoistStepConfig, NativeMoistLargeStep,
                                 upload, weisman_klemp_initial_state)
from gm1_b200.restart import RestartRefusal, read_envelope, resume, write_restart

pytestmark = pytest.mark.gpu

CASES = {
    "python-uniform": (MoistLargeStep, MoistStepConfig(24, 20, 16, 1000.0, 1000.0, 250.0, 5.0, 10),
                       dict(seed=7, bubble_radius_m=(6000.0, 1400.0), bubble_cloud=1.0e-3, bubble_rain=5.0e-4)),
    "native-stretched": (NativeMoistLargeStep,
                         MoistStepConfig(40, 32, 80, 100.0, 100.0, 100.0, 0.6, 8, column=SUPERCELL_STRETCHED_COLUMN),
                         dict(seed=7, bubble_radius_m=(1500.0, 800.0), bubble_center_z_m=800.0, bubble_cloud=1.0e-3,
                              bubble_rain=5.0e-4)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_resumed_run_is_word_identical(tmp_path, case):
    kind, cfg, init = CASES[case]
    host, metrics = weisman_klemp_initial_state(cfg, **init)
    run = kind(cfg, upload(host), upload(metrics))
    for _ in range(3):
        run.step()
    p = tmp_path / "restart.cm1fcp"
    header = write_restart(p, run)
    assert header["step"] == 3 and header["model_time_s"] == 3 * cfg.dt
    for _ in range(3):
        run.step()
    again = kind(cfg, upload(host), upload(metrics))
    resume(again, p)
    assert again.completed_steps == 3
    for _ in range(3):
        again.step()
    torch.cuda.synchronize()
    assert again.completed_steps == run.completed_steps == 6
    differ = [n for n, t in run.s.items()
              if not np.array_equal(t.cpu().numpy().view(np.uint8), again.s[n].cpu().numpy().view(np.uint8))]
    assert not differ, f"{case}: {differ} differ after the resume"
    assert float(run.s["rain"].max()) > 0.0 or float(run.s["q3d"][2].max()) > 0.0


def test_resume_refusals(tmp_path):
    kind, cfg, init = CASES["python-uniform"]
    host, metrics = weisman_klemp_initial_state(cfg, **init)
    run = kind(cfg, upload(host), upload(metrics))
    run.step()
    p = tmp_path / "restart.cm1fcp"
    write_restart(p, run)
    _, arrays = read_envelope(p)
    assert np.array_equal(arrays["u3d"], run.s["u3d"].cpu().numpy())
    other = MoistStepConfig(24, 20, 16, 1000.0, 1000.0, 250.0, 4.0, 10)
    with pytest.raises(RestartRefusal, match="configuration"):
        resume(kind(other, upload(host), upload(metrics)), p)
    changed = kind(cfg, upload(host), upload(metrics))
    changed.s["th0"][3] += 0.5
    with pytest.raises(RestartRefusal, match="base state"):
        resume(changed, p)
