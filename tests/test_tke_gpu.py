"""Parity of the CUDA SGS/TKE local algebra (through the C ABI) with the
reference's CPU twin (golden vectors) and the oracle, under the tolerance
stated in tests/tke_common.py."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.tke import launch_cuda_sgs_tke
from oracle import tke as to
from tests._golden import load_npz
from tests.test_oracle_tke import TAGS
from tests.tke_common import assert_sgs_close

pytestmark = pytest.mark.gpu


def run_gpu(inputs, meta):
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in inputs.items()}
    clip = torch.zeros(1, dtype=torch.int32, device="cuda")
    launch_cuda_sgs_tke(d, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dx=meta["dx"], dy=meta["dy"],
                        dz=meta["dz"], clip_count=clip)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in d.items()}, int(clip.item())


@pytest.mark.parametrize("tag", TAGS)
def test_sgs_tke_matches_reference(tag):
    meta, inputs, out = load_npz(tag)
    got, clipped = run_gpu(inputs, meta)
    assert clipped == meta["clipped"]
    assert_sgs_close(out, got)


def test_sgs_tke_large_matches_oracle():
    from tests.golden.make_golden import sgs_tke_fixture

    meta = dict(ni=200, nj=150, nk=48, dx=100.0, dy=100.0, dz=60.0)
    inputs = sgs_tke_fixture(meta["ni"], meta["nj"], meta["nk"], 99)
    want = {k: v.copy() for k, v in inputs.items()}
    clipped = to.sgs_tke(want, **meta)
    got, gclip = run_gpu(inputs, meta)
    assert gclip == clipped
    assert_sgs_close(want, got)
