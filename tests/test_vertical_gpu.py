"""launch_cuda_stretch_z1 on the GPU: the device generator writes the
reference's own profile words (tests/golden/vertical_levels.json) for every
stretch_z 0 and 1 case, rds/rdsf included, and refuses infeasible columns
before launching."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.vertical import PROFILES, StretchZ1Parameters, launch_cuda_stretch_z1
from tests._golden import load_json

pytestmark = pytest.mark.gpu
G = load_json("vertical_levels.json")


@pytest.mark.parametrize("name", sorted(G["cases"]))
def test_device_profiles_are_the_reference_words(name):
    c = G["cases"][name]
    launch = launch_cuda_stretch_z1(StretchZ1Parameters(*c["stretch_parameters"]), device="cuda:0")
    launch.ready_event.synchronize()
    for f in PROFILES:
        got = getattr(launch.grid, f).cpu().numpy().view(np.uint32)
        assert np.array_equal(got, np.array(c[f], np.uint32)), f
    assert launch.grid.derived.nk2 == c["derived"]["nk2"]


def test_infeasible_column_is_refused_before_launch():
    with pytest.raises(ValueError):
        launch_cuda_stretch_z1(StretchZ1Parameters(75, 100.0, 15000.0, 200.0, 7000.0, 30.0, 320.0), device="cuda:0")
    torch.cuda.synchronize()
