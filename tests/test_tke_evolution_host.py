"""Host-side checks of gm1_b200.tke_evolution: shapes and the reference's
refusals (src/cm1core/cuda_tke_evolution.py:82-96, :437, :449, :481-492),
raised before any library call."""

from __future__ import annotations

import pytest

from gm1_b200 import tke_evolution as te
from gm1_b200.errors import CM1Refusal


def test_shapes():
    s = te.tke_evolution_shapes(7, 7, 8)
    assert s["tke3d"] == (9, 7, 7) and s["rru"] == (10, 13, 14) and s["rrv"] == (10, 14, 13) and s["rrw"] == (11, 13, 13)


def test_refusals():
    with pytest.raises(CM1Refusal):
        te.launch_cuda_tke_evolution({}, ni=7, nj=7, nk=8)
    with pytest.raises(CM1Refusal):
        te.launch_cuda_tke_diffusion({}, ni=7, nj=7, nk=8, dx=1.0, dy=1.0, dz=1.0, dt=1.0,
                                     selection=te.TkeEvolutionSelection(doimpl=0))
    with pytest.raises(ValueError, match="nk"):
        te.tke_evolution_shapes(7, 7, 7)
    with pytest.raises(ValueError, match="nrk"):
        te.launch_cuda_tke_rk_stage({}, workspace=None, ni=7, nj=7, nk=8, nrk=4, dx=1.0, dy=1.0, dz=1.0, dt=1.0)
    with pytest.raises(ValueError, match="completed_nrk"):
        te.launch_cuda_tke_commit({}, ni=7, nj=7, nk=8, completed_nrk=2)
