"""Parity of the CUDA padded-lane advection (through the C ABI) with the
reference's own CPU twins (golden vectors) and with the oracle for the
whole-domain lateral-side variants.  Bar: every float32 word identical."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.advection import launch_cuda_scalar_advection5, launch_cuda_terrain_mass_flux5
from oracle import advection as adv
from tests._golden import bit_mismatches, load_npz
from tests.test_oracle_advection import TAGS, advection_inputs, mass_flux_inputs

pytestmark = pytest.mark.gpu


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("tag", TAGS)
def test_mass_flux_bit_exact_vs_reference(tag):
    meta, inputs, out = load_npz(tag)
    h = mass_flux_inputs(inputs, meta)
    d = {k: dev(v) for k, v in h.items()}
    metrics = {k: d[k] for k in ("rho0_3d", "rf0", "rgzu", "rgzv", "dzdx", "dzdy", "gz")}
    launch_cuda_terrain_mass_flux5(d, metrics, d["divx"], ni=meta["ni"], nj=meta["nj"], nk=meta["nk"],
                                   dx=meta["dx"], dy=meta["dy"], dz=meta["dz"])
    torch.cuda.synchronize()
    got = {k: d[k].cpu().numpy() for k in ("rru", "rrv", "rrw", "divx")}
    want = {"rru": out["mf_rru"], "rrv": out["mf_rrv"], "rrw": out["mf_rrw"], "divx": out["mf_divx"]}
    assert bit_mismatches(want, got, want) == {}


def run_scalar(h, meta, nrk, weps, lateral_sides=None, write_fluxes=True, chunk=None):
    d = {k: dev(v) for k, v in h.items()}
    fluxes = {"x": d["flux_x"], "y": d["flux_y"], "z": d["flux_z"]}
    launch_cuda_scalar_advection5(
        d["scalar"], {k: d[k] for k in ("rru", "rrv", "rrw")}, {k: d[k] for k in ("c1", "c2", "rr0", "gz")},
        d["divx"], d["tendency"], fluxes, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], nrk=nrk, dx=meta["dx"],
        dy=meta["dy"], dz=meta["dz"], weps=weps, lateral_sides=lateral_sides, write_fluxes=write_fluxes,
        levels_per_chunk=chunk)
    torch.cuda.synchronize()
    return {k: d[k].cpu().numpy() for k in ("tendency", "flux_x", "flux_y", "flux_z")}


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("nrk", [1, 2, 3])
@pytest.mark.parametrize("sname", ["scalar", "qscalar"])
def test_scalar_advection_bit_exact_vs_reference(tag, nrk, sname):
    meta, inputs, out = load_npz(tag)
    key = f"{sname}_nrk{1 if nrk < 3 else 3}"
    got = run_scalar(advection_inputs(inputs, meta, sname), meta, nrk, meta["weps"][sname])
    want = {"flux_x": out[f"{key}_fx"], "flux_y": out[f"{key}_fy"], "flux_z": out[f"{key}_fz"],
            "tendency": out[f"{key}_tend"]}
    assert bit_mismatches(want, got, want) == {}


@pytest.mark.parametrize("sides", [(1, 1, 1, 1), (2, 2, 2, 2), (2, 1, 3, 2), (1, 2, 2, 4)])
@pytest.mark.parametrize("nrk", [1, 3])
def test_whole_domain_lateral_sides_match_oracle(sides, nrk):
    from gm1_b200.advection import scalar_open_boundary_code

    meta, inputs, _ = load_npz(TAGS[0])
    h = advection_inputs(inputs, meta, "scalar")
    want = {k: v.copy() for k, v in h.items()}
    adv.scalar_advection5(want, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], nrk=nrk, dx=meta["dx"], dy=meta["dy"],
                          dz=meta["dz"], weps=meta["weps"]["scalar"], lateral_obc=scalar_open_boundary_code(sides))
    got = run_scalar(h, meta, nrk, meta["weps"]["scalar"], lateral_sides=sides)
    assert bit_mismatches(want, got, ("tendency", "flux_x", "flux_y", "flux_z")) == {}
    assert not np.any(got["tendency"] == np.float32(meta["sentinel"]))


@pytest.mark.parametrize("chunk", [1, 3, 4, 100])
def test_fused_path_without_flux_writes_and_any_chunk_is_identical(chunk):
    meta, inputs, out = load_npz(TAGS[1])
    got = run_scalar(advection_inputs(inputs, meta, "qscalar"), meta, 3, meta["weps"]["qscalar"],
                     write_fluxes=False, chunk=chunk)
    assert bit_mismatches({"tendency": out["qscalar_nrk3_tend"]}, got, ("tendency",)) == {}
    assert np.all(got["flux_x"] == np.float32(meta["sentinel"]))


@pytest.mark.parametrize("flat", [False, True])
@pytest.mark.parametrize("nrk", [1, 3])
@pytest.mark.parametrize("sides", [(2, 2, 2, 2), (1, 2, 3, 4)])
def test_stretched_column_matches_oracle(flat, nrk, sides):
    """launch_cuda_gm1_child_stretched_scalar_advection5 on seeded stretched
    profiles (rdsf per level, or mh per level with rdz) against the oracle
    restatement, word for word."""
    from gm1_b200.advection import (StretchedColumn, launch_cuda_gm1_child_stretched_scalar_advection5,
                                    scalar_open_boundary_code)

    meta, inputs, _ = load_npz(TAGS[0])
    nk = meta["nk"]
    h = advection_inputs(inputs, meta, "scalar")
    rng = np.random.default_rng(5)
    rdsf = np.zeros(nk + 3, np.float32)
    rdsf[1:nk + 1] = (np.float32(1.0) / np.float32(meta["dz"])) * rng.uniform(0.4, 2.5, nk).astype(np.float32)
    mh = rng.uniform(0.3, 3.0, nk + 2).astype(np.float32)
    rdz = float(np.float32(1.0) / np.float32(100.0))
    want = {k: v.copy() for k, v in h.items()}
    adv.scalar_advection5_column(want, ni=meta["ni"], nj=meta["nj"], nk=nk, nrk=nrk, dx=meta["dx"], dy=meta["dy"],
                                 weps=meta["weps"]["scalar"], flat=flat, profile=mh if flat else rdsf, rdz=rdz,
                                 lateral_obc=scalar_open_boundary_code(sides))
    d = {k: dev(v) for k, v in h.items()}
    column = StretchedColumn(flat=True, mh=dev(mh), rdz=rdz) if flat else StretchedColumn(flat=False, rdsf=dev(rdsf))
    launch_cuda_gm1_child_stretched_scalar_advection5(
        d["scalar"], {k: d[k] for k in ("rru", "rrv", "rrw")}, {k: d[k] for k in ("c1", "c2", "rr0", "gz")},
        d["divx"], d["tendency"], {"x": d["flux_x"], "y": d["flux_y"], "z": d["flux_z"]}, column,
        ni=meta["ni"], nj=meta["nj"], nk=nk, nrk=nrk, dx=meta["dx"], dy=meta["dy"], weps=meta["weps"]["scalar"],
        lateral_sides=sides)
    torch.cuda.synchronize()
    got = {k: d[k].cpu().numpy() for k in ("tendency", "flux_x", "flux_y", "flux_z")}
    assert bit_mismatches(want, got, ("tendency", "flux_x", "flux_y", "flux_z")) == {}
