"""C-ABI checks that need no GPU: libgm1b.so loads, exports every entry point
include/gm1b.h declares, keeps the struct field order of the header, computes
the acoustic schedule exactly as the reference, and rejects bad arguments
before touching the device."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from gm1_b200 import _native
from gm1_b200.arrays import ALL_ARRAY_NAMES
from oracle import periodic as orc
from tests._golden import load_json

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> list[str]:
    names = []
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        names += re.findall(r"GM1B_API\s+[\w\s\*]+?\b(gm1b_\w+)\s*\(", text)
    return names


def test_library_loads_and_exports_every_declared_symbol():
    lib = _native.lib()
    names = declared_functions()
    assert len(names) >= 6
    for name in names:
        assert hasattr(lib, name), name
    assert lib.gm1b_abi_version() == _native.ABI_VERSION


def test_struct_field_order_matches_header_and_oracle():
    text = (ROOT / "include" / "gm1b.h").read_text()
    body = text[text.index("typedef struct gm1b_periodic_arrays") : text.index("} gm1b_periodic_arrays;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = re.findall(r"\*\s*(\w+)", body)
    assert tuple(fields) == ALL_ARRAY_NAMES
    assert tuple(n for n, _ in _native.PeriodicArrays._fields_) == ALL_ARRAY_NAMES
    assert orc.NAMES == ALL_ARRAY_NAMES


def _header_fields(name: str) -> list[str]:
    text = (ROOT / "include" / "gm1b.h").read_text()
    body = text[text.index(f"typedef struct {name} {{"):text.index(f"}} {name};")]
    body = re.sub(r"/\*.*?\*/", "", body[body.index("{") + 1:], flags=re.S)
    return re.findall(r"\*\s*(\w+)", body)


def test_whole_step_struct_order_matches_header():
    """gm1b_moist_state / gm1b_moist_metrics field order of the header and
    the Python binding of the whole-step entry point, and the config layout."""
    from gm1_b200.moist_step import NATIVE_METRIC_NAMES, NATIVE_STATE_NAMES, _NativeConfig

    assert _header_fields("gm1b_moist_state") == list(NATIVE_STATE_NAMES)
    assert _header_fields("gm1b_moist_metrics") == list(NATIVE_METRIC_NAMES)
    assert ctypes.sizeof(_NativeConfig) == 4 * (3 + 4 + 1 + 2 + 4 + 7)


def test_whole_step_entry_rejects_bad_arguments_without_a_device():
    from gm1_b200.moist_step import _native_lib

    lib = _native_lib()
    handle = ctypes.c_void_p()
    assert lib.gm1b_moist_step_create(None, None, None, ctypes.byref(handle)) == _native.GM1B_ERR_ARGUMENT
    assert lib.gm1b_moist_large_step(None, None) == _native.GM1B_ERR_ARGUMENT
    assert b"NULL" in lib.gm1b_last_error()


def test_schedule_matches_reference_table():
    lib = _native.lib()
    for dt, nsound, nrk, nloop, dts in load_json("schedule.json"):
        n = ctypes.c_int32()
        d = ctypes.c_float()
        assert lib.gm1b_sound3_stage_schedule(dt, nsound, nrk, ctypes.byref(n), ctypes.byref(d)) == 0
        assert (n.value, d.value) == (nloop, dts)
        want = orc.rk_stage_dt(dt, nrk)
        assert lib.gm1b_rk_stage_dt(dt, nrk) == want


@pytest.mark.parametrize("nsound,nrk", [(5, 1), (2, 1), (6, 0), (6, 4)])
def test_schedule_rejects_bad_arguments(nsound, nrk):
    lib = _native.lib()
    n = ctypes.c_int32()
    d = ctypes.c_float()
    assert lib.gm1b_sound3_stage_schedule(6.0, nsound, nrk, ctypes.byref(n), ctypes.byref(d)) == -2
    assert b"nsound" in lib.gm1b_last_error()


def test_entry_points_reject_bad_arguments_without_a_device():
    lib = _native.lib()
    s = _native.PeriodicArrays()  # all NULL
    assert lib.gm1b_psolver3_trajectory(64, 64, 40, None, 1, 6.0, 6, 1e3, 1e3, 500.0, 0, 0, None) == -1
    assert lib.gm1b_psolver3_trajectory(4, 64, 40, ctypes.byref(s), 1, 6.0, 6, 1e3, 1e3, 500.0, 0, 0, None) == -1
    assert lib.gm1b_psolver3_trajectory(64, 64, 40, ctypes.byref(s), 1, 6.0, 7, 1e3, 1e3, 500.0, 0, 0, None) == -2
    assert lib.gm1b_psolver3_trajectory(64, 64, 40, ctypes.byref(s), 1, -6.0, 6, 1e3, 1e3, 500.0, 0, 0, None) == -1
    assert lib.gm1b_psolver3_trajectory(64, 64, 40, ctypes.byref(s), 1, 6.0, 6, 1e3, 1e3, 500.0, 0, 0, None) == -1
    assert b"NULL" in lib.gm1b_last_error()
    assert lib.gm1b_sound3_periodic_three_stage(5, 4, 7, ctypes.byref(s), 2.0, 6, 1e-3, 1e-3, 2e-3,
                                                1005.7, 0.6, 0.1, 0, None) == -1


def test_python_mirror_validates_like_the_reference():
    from gm1_b200.periodic import launch_cuda_psolver3_trajectory, sound3_stage_schedule_f32

    with pytest.raises(ValueError, match="even nsound"):
        sound3_stage_schedule_f32(6.0, 7, 1)
    with pytest.raises(ValueError, match="nrk"):
        sound3_stage_schedule_f32(6.0, 6, 4)
    with pytest.raises(ValueError, match="steps"):
        launch_cuda_psolver3_trajectory({}, ni=8, nj=8, nk=8, steps=0, dt=1.0, nsound=6, dx=1.0, dy=1.0, dz=1.0)
    with pytest.raises(ValueError, match="ni >= 5"):
        launch_cuda_psolver3_trajectory({}, ni=4, nj=8, nk=8, steps=1, dt=1.0, nsound=6, dx=1.0, dy=1.0, dz=1.0)
    with pytest.raises(ValueError, match="missing"):
        launch_cuda_psolver3_trajectory({}, ni=8, nj=8, nk=8, steps=1, dt=1.0, nsound=6, dx=1.0, dy=1.0, dz=1.0)
