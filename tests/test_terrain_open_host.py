"""Host-side contract of the terrain/open acoustic-stage mirror (no GPU):
shapes, selection refusals, ablation masks, the raw-bit comparator and the
launcher's refusals before any device work."""

from __future__ import annotations

import numpy as np
import pytest

from gm1_b200 import terrain_open as tos
from gm1_b200.errors import CM1Refusal
from oracle import terrain_open as orc


def test_shapes_preserve_native_families():
    s = tos.terrain_open_sound_shapes(5, 4, 5)
    assert s["pp3d"] == (7, 6, 7) and s["u3d"] == (7, 10, 12) and s["v3d"] == (7, 11, 11) and s["w3d"] == (8, 10, 11)
    assert set(s) == set(tos.ALL_ARRAY_NAMES) and len(tos.ALL_ARRAY_NAMES) == 45
    assert tos.ALL_ARRAY_NAMES == orc.ARRAY_NAMES
    assert tos.terrain_static_shapes(ni=5, nj=4, nk=5)["gyv"] == (6, 5, 5)


def test_ablation_bits_match_the_oracle():
    for name in orc.ABLATION_BITS:
        assert tos._ablation_mask(tos.TerrainOpenSoundAblations(**{name: False})) == orc.ablation_mask(**{name: False})
    assert tos._ablation_mask(tos.TerrainOpenSoundAblations()) == 255


@pytest.mark.parametrize("field,value,code", [("psolver", 2, "CM1-TERRAIN-OPEN-UNSUPPORTED"),
                                              ("west_boundary", 1, "CM1-TERRAIN-OPEN-UNSUPPORTED"),
                                              ("terrain", 1, "CM1-TERRAIN-OPEN-UNSUPPORTED"),
                                              ("product_admission", True, "CM1-TERRAIN-PRODUCT-SEAM-MISSING")])
def test_selection_refusals(field, value, code):
    with pytest.raises(CM1Refusal) as e:
        tos.validate_terrain_open_selection(tos.TerrainOpenSelection(**{field: value}))
    assert e.value.code == code


def test_comparator_raw_bits():
    a = {n: np.zeros((2, 2), np.float32) for n in tos.COMPARE_OUTPUT_NAMES}
    b = {n: v.copy() for n, v in a.items()}
    assert tos.compare_psolver3_terrain_open_raw(a, b)["passed"]
    b["ppd"][0, 0] = np.float32(-0.0)
    assert not tos.compare_psolver3_terrain_open_raw(a, b)["passed"]
    del b["rrw"]
    with pytest.raises(ValueError, match="rrw"):
        tos.compare_psolver3_terrain_open_raw(a, b)


def test_launcher_refuses_before_device_work():
    kw = dict(ni=5, nj=4, nk=5, dt=0.6, nsound=6, dx=100.0, dy=100.0, dz=200.0)
    with pytest.raises(CM1Refusal):
        tos.launch_cuda_psolver3_terrain_open_three_stage({}, {}, lateral=object(), **kw)
    with pytest.raises(CM1Refusal):
        tos.launch_cuda_psolver3_terrain_open_three_stage({}, {}, nest_substep=object(), **kw)
    with pytest.raises(ValueError, match="alph"):
        tos.launch_cuda_psolver3_terrain_open_three_stage({}, {}, alph=1.5, **kw)
    with pytest.raises(ValueError, match="dz"):
        tos.launch_cuda_psolver3_terrain_open_three_stage({}, {}, **{**kw, "dz": 0.0})
    with pytest.raises(ValueError, match="nrk"):
        tos.launch_cuda_psolver3_terrain_open_stage({}, {}, nrk=4, **kw)
    with pytest.raises(TypeError, match="ablations"):
        tos.launch_cuda_psolver3_terrain_open_three_stage({}, {}, ablations="none", **kw)
