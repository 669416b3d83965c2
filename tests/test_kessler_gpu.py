"""Parity of the CUDA Kessler operator (through the C ABI) with the
reference's own CPU twin (golden vectors) and with the oracle, under the
tolerances stated in tests/kessler_common.py."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.kessler import Gm1KesslerDriverSelection, launch_cuda_gm1_kessler_driver
from oracle import kessler as ko
from tests._golden import load_npz
from tests.kessler_common import assert_budgets_close, assert_fields_close
from tests.test_oracle_kessler import TAGS

pytestmark = pytest.mark.gpu


def run_gpu(inputs, meta):
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in inputs.items()}
    it = torch.zeros((meta["nk"], meta["nj"], meta["ni"]), dtype=torch.int32, device="cuda")
    nf = torch.zeros((meta["nj"], meta["ni"]), dtype=torch.int32, device="cuda")
    launch = launch_cuda_gm1_kessler_driver(
        d, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dx=meta["dx"], dy=meta["dy"], dz=meta["dz"], dt=meta["dt"],
        selection=Gm1KesslerDriverSelection(equation_set=meta["eqtset"]), satadj_iterations=it, nfall=nf)
    status = launch.check()
    got = {k: v.cpu().numpy() for k, v in d.items()}
    return got, it.cpu().numpy().view(np.uint32), nf.cpu().numpy(), status


@pytest.mark.parametrize("tag", TAGS)
def test_kessler_matches_reference(tag):
    meta, inputs, out = load_npz(tag)
    got, it, _, status = run_gpu(inputs, meta)
    assert status["max_fall_substeps"] == meta["max_fall_substeps"]
    assert np.array_equal(it, out["satadj_iterations"])
    assert_fields_close(out, got)
    assert np.array_equal(got["asq"].view(np.uint64), out["asq"].view(np.uint64))
    assert_budgets_close(out["qbudget"], got["qbudget"])


@pytest.mark.parametrize("tag", TAGS)
def test_kessler_matches_oracle_and_is_repeatable(tag):
    meta, inputs, _ = load_npz(tag)
    want = {k: v.copy() for k, v in inputs.items()}
    nf_want = np.zeros((meta["nj"], meta["ni"]), np.int32)
    it_want = np.zeros((meta["nk"], meta["nj"], meta["ni"]), np.uint32)
    ko.kessler_driver(want, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dx=meta["dx"], dy=meta["dy"],
                      dz=meta["dz"], dt=meta["dt"], eqtset=meta["eqtset"], iterations=it_want, nfall=nf_want)
    got, it, nf, _ = run_gpu(inputs, meta)
    again, _, _, _ = run_gpu(inputs, meta)
    assert np.array_equal(nf, nf_want)
    assert np.array_equal(it, it_want)
    assert_fields_close(want, got)
    for k in got:  # run-to-run bit reproducibility (fixed-order reductions)
        assert np.array_equal(np.ascontiguousarray(got[k]).view(np.uint8), np.ascontiguousarray(again[k]).view(np.uint8)), k


def test_kessler_large_domain_matches_oracle():
    """A 96x64x40 domain exercises many CTAs and budget partials."""
    from tests.golden.make_golden import kessler_fixture

    ni, nj, nk, dz, dt = 96, 64, 40, 100.0, 20.0
    inputs = kessler_fixture(ni, nj, nk, dz, 77)
    meta = dict(ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=dz, dt=dt, eqtset=2)
    want = {k: v.copy() for k, v in inputs.items()}
    ko.kessler_driver(want, ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=dz, dt=dt, eqtset=2)
    got, _, _, _ = run_gpu(inputs, meta)
    assert_fields_close(want, got)
    assert np.array_equal(got["asq"].view(np.uint64), want["asq"].view(np.uint64))
    assert_budgets_close(want["qbudget"], got["qbudget"])


def test_fallout_substeps_are_bounded_on_a_blown_up_column():
    """A fall Courant number of about 1.5e7 (rain at 1 kg/kg falling through
    1 m layers over a 1e6 s step) would take int(crmax + 1) sub-steps; the
    operator counts such columns in its third status word, steps them once
    and check() refuses.  Every other column keeps its normal sub-steps."""
    from tests.golden.make_golden import kessler_fixture

    ni, nj, nk = 16, 8, 10
    inputs = kessler_fixture(ni, nj, nk, 100.0, 5)
    inputs["qr"][:, 3, 4] = np.float32(1.0)
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in inputs.items()}
    nf = torch.zeros((nj, ni), dtype=torch.int32, device="cuda")
    launch = launch_cuda_gm1_kessler_driver(d, ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=1.0, dt=1.0e6,
                                            selection=Gm1KesslerDriverSelection(equation_set=2), nfall=nf)
    status = launch.status()
    assert status["blown_up_fall_columns"] >= 1
    assert int(nf[3, 4]) == 1
    with pytest.raises(RuntimeError, match="fall Courant"):
        launch.check()


def nonconvergent_fixture(ni, nj, nk, seed=0):
    """Kessler driver inputs with one cell the saturation adjustment cannot
    settle within its 100 passes: 27.5 % vapour and some cloud at 270 K and
    Exner 0.964 (about 880 hPa), whose given density is the dry density of
    that pressure and temperature.  The driver takes rho and prs as inputs,
    so the state is admissible; the iteration's pressure then disagrees with
    its saturation pressure.  Mixing ratios from 0.265 to 0.285 all run to
    the bound in the oracle, so the cell does not sit on a knife edge."""
    from tests.golden.make_golden import kessler_fixture

    a = kessler_fixture(ni, nj, nk, 100.0, seed)
    k, j, i = 1, nj // 2, ni // 2
    t, pi = 270.0, 0.96388626
    a["qr"][:, j, i] = np.float32(0.0)
    a["pp3d"][k, j, i] = np.float32(pi - a["pi0"][k, j, i])
    a["th3d"][k, j, i] = np.float32(t / pi - a["th0"][k, j, i])
    prs = 1.0e5 * np.float64(pi) ** (1005.7 / 287.04)
    a["prs"][k, j, i] = np.float32(prs)
    a["rho"][k, j, i] = np.float32(prs / (287.04 * t))
    a["qv"][k, j, i] = np.float32(0.275)
    a["qc"][k, j, i] = np.float32(6.0e-3)
    return a, (k, j, i)


def test_satadj_nonconvergence_is_counted_like_the_oracle():
    """The non-converging cell takes the full 100 passes on the GPU as in the
    oracle, the status word counts it and check() refuses it as the
    reference does."""
    ni, nj, nk = 8, 8, 4
    a, cell = nonconvergent_fixture(ni, nj, nk)
    it_want = np.zeros((nk, nj, ni), np.uint32)
    want = {k: v.copy() for k, v in a.items()}
    with pytest.raises(RuntimeError, match="converge"):
        ko.kessler_driver(want, ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=100.0, dt=5.0, eqtset=2,
                          iterations=it_want)
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in a.items()}
    it = torch.zeros((nk, nj, ni), dtype=torch.int32, device="cuda")
    launch = launch_cuda_gm1_kessler_driver(d, ni=ni, nj=nj, nk=nk, dx=1000.0, dy=1000.0, dz=100.0, dt=5.0,
                                            selection=Gm1KesslerDriverSelection(equation_set=2),
                                            satadj_iterations=it)
    status = launch.status()
    got = it.cpu().numpy().view(np.uint32)
    assert got[cell] == 100 and it_want[cell] == 100
    assert status["satadj_nonconverged_cells"] == int(np.count_nonzero(it_want >= 100))
    with pytest.raises(RuntimeError, match="converge"):
        launch.check()
