"""Host-side behaviour of the Kessler operator API (no GPU needed)."""

from __future__ import annotations

import pytest

from gm1_b200.errors import CM1Refusal
from gm1_b200.kessler import Gm1KesslerDriverSelection, gm1_kessler_driver_shapes, launch_cuda_gm1_kessler_driver


@pytest.mark.parametrize("field,value,code", [("efall", 1, "GM1-KESSLER-DRIVER-EFALL"),
                                              ("equation_set", 3, "GM1-KESSLER-DRIVER-EQTSET"),
                                              ("ptype", 2, "GM1-KESSLER-DRIVER-SELECTION"),
                                              ("rain_bins", 2, "GM1-KESSLER-DRIVER-SELECTION")])
def test_unsupported_selections_are_refused(field, value, code):
    with pytest.raises(CM1Refusal) as info:
        launch_cuda_gm1_kessler_driver({}, ni=4, nj=4, nk=4, dx=1.0, dy=1.0, dz=1.0, dt=1.0,
                                       selection=Gm1KesslerDriverSelection(**{field: value}))
    assert info.value.code == code


def test_shapes_and_argument_checks():
    s = gm1_kessler_driver_shapes(5, 4, 3)
    assert s["qv"] == (3, 4, 5) and s["rain"] == (1, 4, 5) and s["prate"] == (4, 5) and s["qbudget"] == (10,)
    with pytest.raises(ValueError, match="missing"):
        launch_cuda_gm1_kessler_driver({}, ni=4, nj=4, nk=4, dx=1.0, dy=1.0, dz=1.0, dt=1.0)
    with pytest.raises(ValueError, match="dt"):
        launch_cuda_gm1_kessler_driver({}, ni=4, nj=4, nk=4, dx=1.0, dy=1.0, dz=1.0, dt=0.0)


def test_c_abi_rejects_bad_kessler_arguments_without_a_device():
    import ctypes

    from gm1_b200.kessler import _bind, _KesslerArrays

    lib = _bind()
    s = _KesslerArrays()
    assert lib.gm1b_kessler_workspace_bytes(64, 64, 40) > 16
    assert lib.gm1b_kessler_driver(8, 8, 8, ctypes.byref(s), 1.0, 1.0, 1.0, 1.0, 2, 0, None, 0, None) == -1
    assert lib.gm1b_kessler_driver(8, 8, 8, ctypes.byref(s), 1.0, 1.0, 1.0, 1.0, 2, 1, None, 0, None) == -1
    assert b"efall" in lib.gm1b_last_error()
