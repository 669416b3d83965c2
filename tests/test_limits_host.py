"""Host-side argument checks of gm1_b200.limits: the reference's TypeError /
ValueError refusals (src/cm1core/gm1_runtime.py:259-263, :277-281, :478-486)
are raised before any library call."""

from __future__ import annotations

import math

import pytest

from gm1_b200 import limits


@pytest.mark.parametrize("bad", [0.0, -1.0, math.inf, math.nan])
def test_spacing_refusals(bad):
    with pytest.raises(ValueError, match="finite and positive"):
        limits.cm1_acoustic_small_step_limit_s(dx_m=bad, dy_m=1000.0)
    with pytest.raises(ValueError, match="finite and positive"):
        limits.cm1_diagnostic_acoustic_substeps(dt_s=6.0, dx_m=1000.0, dy_m=bad)


def test_type_refusals():
    with pytest.raises(TypeError):
        limits.cm1_acoustic_small_step_limit_s(dx_m=True, dy_m=1000.0)
    with pytest.raises(TypeError):
        limits.cm1_advective_courant(dt_s=6.0, dx_m=1e3, dy_m=1e3, dz_m=500.0, u_m_s="1", v_m_s=0.0, w_m_s=0.0)
    with pytest.raises(ValueError, match="finite"):
        limits.cm1_advective_courant(dt_s=6.0, dx_m=1e3, dy_m=1e3, dz_m=500.0, u_m_s=math.inf, v_m_s=0.0,
                                     w_m_s=0.0)


def test_courant_factors_are_binary32_in_reference_order():
    import numpy as np  # noqa: PLC0415

    f = np.float32
    dtdx, dtdy, dtdz = limits.courant_factors(dt_s=6.0, dx_m=333.33, dy_m=1000.0, dz_m=250.0)
    assert dtdx == float(f(f(f(0.5) * f(6.0)) * f(1.0 / 333.33)))
    assert dtdz == float(f(f(f(0.5) * f(6.0)) * f(1.0 / 250.0)))
