"""The library's CM1 limits (gm1_b200.limits on libgm1b.so) against the
reference's own outputs (tests/golden/limits_courant.npz) and the oracle.
Bars: every scalar exact (binary64); the domain Courant number and every
per-level maximum word-identical (binary32 cell arithmetic in the
reference's order; max is order-free), NaN and inf levels included."""

from __future__ import annotations

import json

import numpy as np
import pytest
import torch

from gm1_b200.limits import (
    advective_courant_number,
    cm1_acoustic_small_step_limit_s,
    cm1_advective_courant,
    cm1_diagnostic_acoustic_substeps,
)
from oracle import limits as orc
from tests.test_oracle_limits import _cases, factors

pytestmark = pytest.mark.gpu


def test_scalars_match_reference_table():
    _, table, _ = _cases()
    for row in table:
        assert cm1_acoustic_small_step_limit_s(dx_m=row["dx"], dy_m=row["dy"]) == row["limit"]
        assert cm1_diagnostic_acoustic_substeps(dt_s=row["dt"], dx_m=row["dx"], dy_m=row["dy"]) == row["nsound"]
        got = cm1_advective_courant(dt_s=row["dt"], dx_m=row["dx"], dy_m=row["dy"], dz_m=row["dz"], u_m_s=row["u"],
                                    v_m_s=row["v"], w_m_s=row["w"])
        assert got == row["courant"]


@pytest.mark.parametrize("tag", ["a", "b", "c", "d", "e"])
def test_domain_courant_kernel_matches_reference_and_oracle(tag):
    z, _, _ = _cases()
    meta = json.loads(str(z[f"{tag}_meta"]))
    dev = {n: torch.from_numpy(np.ascontiguousarray(z[f"{tag}_{n}"])).cuda() for n in ("u", "v", "w", "uh", "vh", "mh")}
    keys = torch.empty(meta["nz"], dtype=torch.int32, device="cuda")
    out = advective_courant_number(**dev, dt_s=meta["dt"], dx_m=meta["dx"], dy_m=meta["dy"], dz_m=meta["dz"],
                                   level_keys=keys)
    torch.cuda.synchronize()
    got = float(out.cpu()[0])
    want = meta["courant"]
    assert (got == want) or (np.isinf(got) and np.isinf(want))
    _, levels = orc.courant_max(*(z[f"{tag}_{n}"] for n in ("u", "v", "w", "uh", "vh", "mh")), *factors(meta))
    key = keys.cpu().numpy().view(np.uint32)
    want_key = np.where(np.isnan(levels), np.uint32(0xFFFFFFFF), levels.view(np.uint32))
    assert np.array_equal(key, want_key)


def test_domain_courant_large_grid_matches_oracle():
    rng = np.random.default_rng(5)
    nk, nj, ni = 40, 192, 160
    u = rng.normal(10, 15, (nk, nj, ni + 1)).astype(np.float32)
    v = rng.normal(0, 15, (nk, nj + 1, ni)).astype(np.float32)
    w = rng.normal(0, 5, (nk + 1, nj, ni)).astype(np.float32)
    uh = rng.uniform(0.9, 1.1, ni).astype(np.float32)
    vh = rng.uniform(0.9, 1.1, nj).astype(np.float32)
    mh = rng.uniform(0.5, 2.0, nk).astype(np.float32)
    meta = {"dt": 6.0, "dx": 1000.0, "dy": 1000.0, "dz": 250.0}
    want, _ = orc.courant_max(u, v, w, uh, vh, mh, *factors(meta))
    dev = {n: torch.from_numpy(a).cuda() for n, a in (("u", u), ("v", v), ("w", w), ("uh", uh), ("vh", vh), ("mh", mh))}
    out = advective_courant_number(**dev, dt_s=6.0, dx_m=1000.0, dy_m=1000.0, dz_m=250.0)
    assert float(out.cpu()[0]) == want
