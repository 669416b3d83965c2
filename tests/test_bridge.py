"""eqtset=2 stage terms: the oracle against the reference's own cell twin
(cpu_eqtset2_cell_f32) bit for bit, and the CUDA operator against the
golden cells laid out as a 3-D domain (gpu)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import bridge
from tests._golden import GOLDEN


def load():
    with np.load(GOLDEN / "eqtset2_cells.npz") as z:
        return {k[3:]: z[k] for k in z.files if k.startswith("in_")}, z["out_terms"]


def test_eqtset2_cell_oracle_matches_reference():
    inp, out = load()
    for c in range(out.shape[1]):
        got = bridge.eqtset2_cell(inp["th0"][c], inp["qv0"][c], inp["pi0"][c], inp["qc0"][c], inp["qi0"][c],
                                  inp["th3d"][c], inp["pp3d"][c], inp["q"][:, c])
        assert np.array_equal(got.view(np.uint32), out[:, c].view(np.uint32)), c


@pytest.mark.gpu
def test_eqtset2_stage_terms_bit_exact_vs_reference_cells():
    from gm1_b200.moist_bridge import launch_cuda_eqtset2_stage_terms

    inp, out = load()
    nk, nj, ni = 4, 10, 10  # 400 golden cells as a (nk, nj, ni) domain with 3-D base state
    sh = (nk, nj, ni)
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    pp3d = np.zeros((nk + 2, nj + 2, ni + 2), np.float32)
    pp3d[1:-1, 1:-1, 1:-1] = inp["pp3d"].reshape(sh)
    tens = {n: torch.zeros((nk + 2, nj + 2, ni + 2), device="cuda") for n in ("thv", "ppterm", "piadv")}
    buoy = torch.zeros((nk + 2, nj + 6, ni + 6), device="cuda")
    thterm = torch.zeros(sh, device="cuda")
    launch_cuda_eqtset2_stage_terms(ni=ni, nj=nj, nk=nk, th0=d(inp["th0"].reshape(sh)), qv0=d(inp["qv0"].reshape(sh)),
                                    pi0=d(inp["pi0"].reshape(sh)), qc0=d(inp["qc0"].reshape(sh)),
                                    qi0=d(inp["qi0"].reshape(sh)), th3d=d(inp["th3d"].reshape(sh)),
                                    q3d=d(inp["q"].reshape((6,) + sh)), pp3d=d(pp3d), thv=tens["thv"],
                                    ppterm=tens["ppterm"], buoyancy=buoy, thterm=thterm, piadv=tens["piadv"],
                                    base3d=True)
    torch.cuda.synchronize()
    got = np.stack([buoy.cpu().numpy()[1:-1, 3:-3, 3:-3].reshape(-1),
                    tens["thv"].cpu().numpy()[1:-1, 1:-1, 1:-1].reshape(-1),
                    thterm.cpu().numpy().reshape(-1),
                    tens["ppterm"].cpu().numpy()[1:-1, 1:-1, 1:-1].reshape(-1)])
    assert np.array_equal(got.view(np.uint32), out.view(np.uint32))
    piadv = tens["piadv"].cpu().numpy()
    want_piadv = (inp["pi0"].reshape(sh) + inp["pp3d"].reshape(sh)).astype(np.float32)
    assert np.array_equal(piadv[1:-1, 1:-1, 1:-1].view(np.uint32), want_piadv.view(np.uint32))
