"""The flat stretched-column closure kernels on the GPU (through the C ABI)
against golden vectors of the reference's own CUDA texts run on the host
(src/cm1core/cuda_gm1_flat_stretched_closure.py; see
tests/golden/make_kernel_text_golden.py): calcdef, turbt and the three TKE
RK stages, every word identical."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.closure import launch_cuda_flat_deformation
from gm1_b200.tke_evolution import launch_cuda_flat_tke_diffusion, launch_cuda_flat_tke_rk_stage
from tests.test_oracle_flat_closure import CASES, load_flat, same

pytestmark = pytest.mark.gpu


def _dev(a):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in a.items() if isinstance(v, np.ndarray)
            and v.ndim > 0}


@pytest.mark.parametrize("tag", CASES)
def test_flat_calcdef_gpu_matches_reference_text(tag):
    p, a, out = load_flat(tag)
    d = _dev(a)
    d["defv"] = torch.full(out["defv"].shape, 7.0, device="cuda")
    d["defh"] = torch.full(out["defh"].shape, 7.0, device="cuda")
    launch_cuda_flat_deformation(d, mh_profile=d["mh_profile"], ni=p["ni"], nj=p["nj"], nk=p["nk"], dx=p["dx"],
                                 dy=p["dy"], rdz=p["rdz"]).ready_event.synchronize()
    assert same(d["defv"].cpu().numpy(), out["defv"]) and same(d["defh"].cpu().numpy(), out["defh"])


@pytest.mark.parametrize("tag", CASES)
def test_flat_turbt_and_tke_stages_gpu_match_reference_text(tag):
    p, a, out = load_flat(tag)
    d = _dev(a)
    g = dict(ni=p["ni"], nj=p["nj"], nk=p["nk"], dx=p["dx"], dy=p["dy"], rdz=p["rdz"], dt=p["dt"])
    launch_cuda_flat_tke_diffusion(d, **g).ready_event.synchronize()
    assert same(d["tketen"].cpu().numpy(), out["tketen_turbt"])
    ws = torch.zeros_like(d["tke3d"])
    for nrk in (1, 2, 3):
        launch_cuda_flat_tke_rk_stage(d, mf_profile=d["mf_profile"], workspace=ws, nrk=nrk, **g)
        torch.cuda.synchronize()
        assert same(d["tke3d"].cpu().numpy(), out[f"tke_stage{nrk}"]), nrk
