"""The FP64 run of the oracle's composition (oracle/fp64_twin.py): the same
operators evaluated in binary64 stay within the float32 rounding of the
binary32 oracle (each field on its own scale) and are not the binary32
words (the widened build really computes in double precision), on both
column families, from the same float32 starting words."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from oracle.fp64_twin import OUT_FIELDS, run_fp64
from oracle.moist_composition import OracleMoistStep
from oracle.moist_initial import weisman_klemp_initial_state
from tests.moist_common import FIELDS, field_errors, format_errors

STRETCHED = SimpleNamespace(ztop_m=20800.0, str_bot_m=200.0, str_top_m=15800.0, dz_bot_m=20.0, dz_top_m=500.0)


def _start(ni, nj, nk, dx, dz, dt, nsound, column):
    cfg = SimpleNamespace(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, dt=dt, nsound=nsound, alph=0.60, kdiv=0.10,
                          lateral_sides=(2, 2, 2, 2), obc=0x2222, column=column)
    host, metrics = weisman_klemp_initial_state(cfg, seed=3, bubble_radius_m=(4.0 * dx, 4.0 * dz),
                                                bubble_center_z_m=4.0 * dz, bubble_cloud=1.0e-3, bubble_rain=5.0e-4)
    return cfg, host, metrics


@pytest.mark.parametrize("column", [None, STRETCHED], ids=["uniform", "stretched"])
def test_fp64_run_is_the_binary32_composition_widened(column):
    if column is None:
        cfg, host, metrics = _start(16, 12, 12, 1000.0, 250.0, 5.0, 10, None)
    else:
        cfg, host, metrics = _start(12, 10, 80, 100.0, 100.0, 0.6, 8, column)
    f64 = run_fp64(cfg, {k: v.copy() for k, v in host.items()}, {k: v.copy() for k, v in metrics.items()}, 2,
                   snapshots=(1, 2), threads=2)
    ref = OracleMoistStep(cfg, host, metrics)
    for step in (1, 2):
        ref.step()
        got = f64[step]
        assert set(got) == set(OUT_FIELDS) and all(a.dtype == np.float64 for a in got.values())
        err = field_errors(ref.s, got)
        print(step, format_errors(err))
        # within float32 rounding carried through two steps of a convective start
        for n in FIELDS:
            assert err[n][0] <= 1.0e-2 and err[n][1] <= 1.0e-3, (n, step, err[n])
        # and not the binary32 words: the widened build rounds differently
        assert any(not np.array_equal(ref.s[n].astype(np.float64), got[n]) for n in ("w3d", "pp3d", "th3d"))
        assert err["w3d"][0] > 0.0 and err["pp3d"][0] > 0.0
