"""Each float32 prognostic field of the composed moist step against the FP64
run of the same operators (the oracle's composition with every binary32
operation evaluated in binary64, oracle/fp64_twin.py), after 1 and 10 large
steps, on the uniform column (configuration 2's physics on a 24x20x16 grid)
and on the 80-level stretched supercell column of configuration 3 (48x40
plane; also with the SGS stress, scalar diffusion and Rayleigh damping held
tendencies on),
starts with cloud and rain in the bubble.

Stated tolerance (tests/fp64_common.py): the GPU's error against the FP64
run, each field on its own scale, at most four times the binary32 oracle's
own error against it (the reference algorithm's float32 rounding), plus a
floor of 2e-6 (max) / 2e-7 (RMS) of the field's scale."""

from __future__ import annotations

import pytest

from gm1_b200.moist_step import (SUPERCELL_STRETCHED_COLUMN, MoistLargeStep, MoistStepConfig, upload,
                                 weisman_klemp_initial_state)
from tests.fp64_common import describe, fp64_bars, fp64_errors
from tests.moist_common import check_errors

pytestmark = pytest.mark.gpu


def _gpu(cfg, host, metrics):
    return MoistLargeStep(cfg, upload(host), upload(metrics))


CASES = {
    "uniform-24x20x16": (MoistStepConfig(24, 20, 16, 1000.0, 1000.0, 250.0, 5.0, 10),
                         dict(seed=7, bubble_radius_m=(6000.0, 1400.0), bubble_cloud=1.0e-3, bubble_rain=5.0e-4)),
    "stretched-48x40x80": (MoistStepConfig(48, 40, 80, 100.0, 100.0, 100.0, 0.6, 8, column=SUPERCELL_STRETCHED_COLUMN),
                           dict(seed=7, bubble_radius_m=(1500.0, 800.0), bubble_center_z_m=800.0,
                                bubble_cloud=1.0e-3, bubble_rain=5.0e-4)),
    # the same column with the closure's held tendencies (SGS stress, scalar
    # diffusion, upper Rayleigh damping, dissipative heating)
    "stretched-48x40x80-held": (MoistStepConfig(48, 40, 80, 100.0, 100.0, 100.0, 0.6, 8,
                                                column=SUPERCELL_STRETCHED_COLUMN, sgs_diffusion=True,
                                                rayleigh=True, dissipative_heating=True),
                               dict(seed=7, bubble_radius_m=(1500.0, 800.0), bubble_center_z_m=800.0,
                                    bubble_cloud=1.0e-3, bubble_rain=5.0e-4)),
    # the uniform column's terrain texts of the stress and turbs, with the
    # damping layer brought down into its 4 km
    "uniform-24x20x16-held": (MoistStepConfig(24, 20, 16, 1000.0, 1000.0, 250.0, 5.0, 10, sgs_diffusion=True,
                                              rayleigh=True, dissipative_heating=True, rayleigh_zd_m=3000.0),
                              dict(seed=7, bubble_radius_m=(6000.0, 1400.0), bubble_cloud=1.0e-3,
                                   bubble_rain=5.0e-4)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_error_against_fp64_run_matches_the_oracles(case):
    cfg, init = CASES[case]
    host, metrics = weisman_klemp_initial_state(cfg, **init)
    errs = fp64_errors(cfg, host, metrics, (1, 10), _gpu)
    print(case, describe(errs))
    for step, (gpu, oracle) in errs.items():
        check_errors(gpu, fp64_bars(oracle), f"{case} step {step} against the FP64 run")
