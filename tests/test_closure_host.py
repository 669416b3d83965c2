"""Host-side checks of gm1_b200.closure: shapes and the reference's refusals
(src/cm1core/cuda_terrain_deformation.py:88-127, src/cm1core/cuda_moist_nm.py:70-104),
raised before any library call."""

from __future__ import annotations

import pytest

from gm1_b200 import closure
from gm1_b200.errors import CM1Refusal


def test_shapes_match_reference():
    s = closure.terrain_deformation_shapes(4, 3, 5)
    assert s["defv"] == (6, 3, 4) and s["u3d"] == (5, 3, 5) and s["rgzv"] == (4, 4)
    m = closure.moist_nm_array_shapes(4, 3, 5)
    assert m["q3d"] == (6, 5, 3, 4) and m["nm"] == (6, 3, 4) and m["pi0"] == (5,)


def test_refusals():
    with pytest.raises(CM1Refusal):
        closure.launch_cuda_terrain_deformation({}, ni=4, nj=4, nk=4, dx=1.0, dy=1.0, dz=1.0,
                                                selection=closure.TerrainDeformationSelection(axisymmetric=1))
    with pytest.raises(CM1Refusal):
        closure.launch_cuda_moist_nm({}, ni=4, nj=4, nk=4, dz=1.0, selection=closure.MoistNmSelection(numq=3))
    with pytest.raises(ValueError):
        closure.terrain_deformation_shapes(2, 4, 4)
    with pytest.raises(ValueError, match="missing"):
        closure.launch_cuda_moist_nm({}, ni=4, nj=4, nk=4, dz=1.0)
    with pytest.raises(ValueError, match="finite"):
        closure.launch_cuda_terrain_deformation({}, ni=4, nj=4, nk=4, dx=0.0, dy=1.0, dz=1.0)
