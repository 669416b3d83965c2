"""Host-side behaviour of the advection operator API (no GPU needed)."""

from __future__ import annotations

import pytest

from gm1_b200.advection import (
    Advection5Selection,
    launch_cuda_scalar_advection5,
    scalar_advection_uses_weno,
    scalar_open_boundary_code,
)
from gm1_b200.errors import CM1Refusal


def test_weno_selected_only_on_final_stage():
    assert [scalar_advection_uses_weno(n) for n in (1, 2, 3)] == [False, False, True]
    assert scalar_advection_uses_weno(3, wflag=False) is False
    with pytest.raises(ValueError):
        scalar_advection_uses_weno(4)


@pytest.mark.parametrize("field,value", [("velocity_weno", 2), ("positive_definite", True), ("weno_order", 3),
                                         ("mpi", True)])
def test_unsupported_branches_are_refused(field, value):
    with pytest.raises(CM1Refusal) as info:
        scalar_advection_uses_weno(3, selection=Advection5Selection(**{field: value}))
    assert info.value.code == "CM1-ADVECTION5-UNSUPPORTED"


def test_lateral_side_codes():
    assert scalar_open_boundary_code(None) == 0
    assert scalar_open_boundary_code((1, 1, 1, 1)) == 0x1111
    assert scalar_open_boundary_code((2, 1, 3, 4)) == 2 | (1 << 4) | (3 << 8) | (4 << 12)
    with pytest.raises(ValueError):
        scalar_open_boundary_code((0, 1, 1, 1))


def test_bad_arguments_are_rejected_before_any_launch():
    kw = dict(ni=16, nj=16, nk=16, nrk=1, dx=1.0, dy=1.0, dz=1.0, weps=1e-6)
    with pytest.raises(ValueError, match="weps"):
        launch_cuda_scalar_advection5(None, {}, {}, None, None, None, **{**kw, "weps": 0.0})
    with pytest.raises(ValueError, match="ni"):
        launch_cuda_scalar_advection5(None, {}, {}, None, None, None, **{**kw, "ni": 4})
    with pytest.raises(TypeError):
        launch_cuda_scalar_advection5(None, {}, {}, None, None, None, **kw)
