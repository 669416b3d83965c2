"""Pins the padded-lane advection oracle to the reference's own CPU twins
(cpu_terrain_mass_flux5_inplace, cpu_scalar_advection5_inplace) word for
word, on golden fixtures with both flux signs and signed zeros."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import advection as adv
from tests._golden import bit_mismatches, load_npz

TAGS = ["adv5_12x10x9", "adv5_9x11x10"]


def mass_flux_inputs(inputs, meta):
    s = meta["sentinel"]
    a = {n: inputs[n].copy() for n in ("u3d", "v3d", "w3d", "rho0_3d", "rf0", "rgzu", "rgzv", "dzdx", "dzdy", "gz")}
    a["rru"] = np.full_like(inputs["u3d"], np.float32(s))
    a["rrv"] = np.full_like(inputs["v3d"], np.float32(s))
    a["rrw"] = np.full_like(inputs["w3d"], np.float32(s))
    a["divx"] = np.full_like(inputs["rr0"], np.float32(s))
    return a


def advection_inputs(inputs, meta, sname):
    s = meta["sentinel"]
    return {
        "scalar": inputs[sname].copy(), "rru": inputs["adv_rru"].copy(), "rrv": inputs["adv_rrv"].copy(),
        "rrw": inputs["adv_rrw"].copy(), "c1": inputs["c1"].copy(), "c2": inputs["c2"].copy(),
        "rr0": inputs["rr0"].copy(), "gz": inputs["gz"].copy(), "divx": inputs["adv_divx"].copy(),
        "tendency": np.full_like(inputs["rr0"], np.float32(s)),
        "flux_x": np.full_like(inputs["adv_rru"], np.float32(s)),
        "flux_y": np.full_like(inputs["adv_rrv"], np.float32(s)),
        "flux_z": np.full_like(inputs["adv_rrw"], np.float32(s)),
    }


@pytest.mark.parametrize("tag", TAGS)
def test_mass_flux_oracle_matches_reference(tag):
    meta, inputs, out = load_npz(tag)
    a = mass_flux_inputs(inputs, meta)
    adv.terrain_mass_flux5(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dx=meta["dx"], dy=meta["dy"], dz=meta["dz"])
    want = {"rru": out["mf_rru"], "rrv": out["mf_rrv"], "rrw": out["mf_rrw"], "divx": out["mf_divx"]}
    assert bit_mismatches(want, a, want) == {}


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("nrk", [1, 3])
@pytest.mark.parametrize("sname", ["scalar", "qscalar"])
def test_scalar_advection_oracle_matches_reference(tag, nrk, sname):
    meta, inputs, out = load_npz(tag)
    a = advection_inputs(inputs, meta, sname)
    adv.scalar_advection5(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], nrk=nrk, dx=meta["dx"], dy=meta["dy"],
                          dz=meta["dz"], weps=meta["weps"][sname])
    key = f"{sname}_nrk{nrk}"
    want = {"flux_x": out[f"{key}_fx"], "flux_y": out[f"{key}_fy"], "flux_z": out[f"{key}_fz"],
            "tendency": out[f"{key}_tend"]}
    assert bit_mismatches(want, a, want) == {}


def test_weno_only_on_final_stage_changes_tendency():
    """WENO is selected only at nrk = 3 (reference test_cuda_advection5.py:149-197)."""
    meta, inputs, out = load_npz(TAGS[0])
    t1, t3 = out["scalar_nrk1_tend"], out["scalar_nrk3_tend"]
    assert not np.array_equal(t1.view(np.uint32), t3.view(np.uint32))
    ring = np.ones_like(t1, dtype=bool)
    ring[:, 3:-3, 3:-3] = False
    assert np.all(t1[ring] == np.float32(meta["sentinel"]))
