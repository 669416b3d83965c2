"""The final-RK dry-air mass correction on the GPU (gm1b_apmasscon,
gm1b_dry_mass, gm1b_kessler_large_step_apmasscon):

* against the reference's CPU twin (golden apmasscon_*.npz): the binary64
  ledgers (one CTA per level, a fixed tree order, against the twin's serial
  sums) within 1e-13 relative, the binary32 correction and pp3d word-identical,
  prs and rho within 2 ulp (powf), the diagnostics words in order;
* the initial ledger of the starting state against the twin's mass1;
* the Kessler large step with the correction between the pre-physics
  equation of state and the driver, over two transitions, against the
  oracle's under the Kessler tolerances (the ledger within 1e-8 and the
  correction within 1e-5 relative: they sum densities whose words carry
  powf ulps);
* the moist step's ledger is taken once, from its starting state, and kept
  when the state already holds one (a restored ledger)."""

from __future__ import annotations

import json

import numpy as np
import pytest
import torch

from gm1_b200 import kessler as gk
from oracle import kessler as ko
from tests._golden import GOLDEN
from tests.golden.make_golden import APMASSCON_CASES, apmasscon_fixture, kessler_large_step_fixture
from tests.kessler_common import assert_fields_close
from tests.test_oracle_kessler_large_step import assert_held_close

pytestmark = pytest.mark.gpu

TAGS = ("apmasscon_9x7x12", "apmasscon_13x6x10")


def _dev(d):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in d.items()}


def _ulps(a, b):
    return int(np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64)).max())


@pytest.mark.parametrize("tag", TAGS)
def test_correction_matches_the_reference_twin(tag):
    z = np.load(GOLDEN / f"{tag}.npz")
    meta = json.loads(str(z["meta"]))
    ni, nj, nk = meta["ni"], meta["nj"], meta["nk"]
    a = _dev({n: z[f"in_{n}"] for n in gk.APMASSCON_ARRAY_NAMES})
    r = gk.launch_cuda_apmasscon(a, ni=ni, nj=nj, nk=nk, mass1=meta["mass1"])
    r.ready_event.synchronize()
    d = r.diagnostics.cpu().numpy()
    assert abs(d[0] - meta["mass2"]) <= 1e-13 * meta["mass2"]
    assert abs(d[1] - meta["pressure_sum"]) <= 1e-13 * meta["pressure_sum"]
    assert np.float32(d[2]) == np.float32(meta["correction"]) and d[3] == meta["mass1"]
    assert np.array_equal(a["pp3d"].cpu().numpy().view(np.uint32), z["out_pp3d"].view(np.uint32))
    for n in ("prs", "rho"):
        assert _ulps(a[n].cpu().numpy(), z[f"out_{n}"]) <= 2, n


@pytest.mark.parametrize("tag", TAGS)
def test_initial_ledger_matches_the_reference_twin(tag):
    meta = json.loads(str(np.load(GOLDEN / f"{tag}.npz")["meta"]))
    ni, nj, nk = meta["ni"], meta["nj"], meta["nk"]
    start = _dev(apmasscon_fixture(ni, nj, nk, APMASSCON_CASES[tag][3]))
    m = gk.dry_mass(start["rho"], start["ruh"], start["rvh"], start["rmh"], ni=ni, nj=nj, nk=nk)
    assert abs(float(m.item()) - meta["mass1"]) <= 1e-13 * meta["mass1"]
    kept = torch.tensor([123.5], dtype=torch.float64, device="cuda")
    gk.dry_mass(start["rho"], start["ruh"], start["rvh"], start["rmh"], ni=ni, nj=nj, nk=nk, out=kept,
                only_if_unset=True)
    assert float(kept.item()) == 123.5


def test_large_step_with_the_correction_matches_the_oracle():
    ni, nj, nk, dz, dt = 40, 33, 30, 120.0, 10.0
    a, held = kessler_large_step_fixture(ni, nj, nk, dz, 78)
    ref_a, ref_h = {k: v.copy() for k, v in a.items()}, {k: v.copy() for k, v in held.items()}
    mass1 = ko.dry_mass(a["rho"], a["ruh"], a["rvh"], a["rmh"], ni=ni, nj=nj, nk=nk) * 0.999
    ref_m1 = np.array([mass1], np.float64)
    dev, hdev = _dev(a), _dev(held)
    m1 = torch.tensor([mass1], dtype=torch.float64, device="cuda")
    t = gk.create_cuda_gm1_kessler_large_step_transition(
        dev, ni=ni, nj=nj, nk=nk, dx=500.0, dy=500.0, dz=dz, dt=dt,
        selection=gk.Gm1KesslerDriverSelection(equation_set=2),
        carriers=gk.Gm1KesslerHeldCarriers(*(hdev[n] for n in gk.HELD_NAMES)), mass1=m1)
    for _ in (1, 2):
        t.apply()
        diag = np.zeros(4, np.float64)
        ko.kessler_large_step(ref_a, ref_h, ni=ni, nj=nj, nk=nk, dx=500.0, dy=500.0, dz=dz, dt=dt, eqtset=2,
                              mass1=ref_m1, mass_diag=diag)
        torch.cuda.synchronize()
        got = {k: v.cpu().numpy() for k, v in t.arrays.items()}
        assert_fields_close(ref_a, got)
        assert_held_close(ref_h, {k: v.cpu().numpy() for k, v in hdev.items()}, ref_a, dt)
        # the ledger sums the pre-physics densities, whose words differ by the
        # powf ulps the Kessler tolerances allow: mass2 agrees to ~1e-9, and
        # the correction, (mass1/mass2)^rddcv - 1 of a 1e-3 drift, to ~1e-6
        d = t.mass_diagnostics.cpu().numpy()
        assert abs(d[0] - diag[0]) <= 1e-8 * diag[0]
        assert diag[2] != 0.0 and abs(d[2] - diag[2]) <= 1e-5 * abs(diag[2])


def test_moist_step_takes_its_ledger_once():
    from gm1_b200.moist_step import MoistLargeStep, MoistStepConfig, upload, weisman_klemp_initial_state  # noqa: PLC0415

    cfg = MoistStepConfig(24, 20, 16, 1000.0, 1000.0, 250.0, 5.0, 10)
    host, metrics = weisman_klemp_initial_state(cfg, seed=7)
    assert host["mass1"][0] == 0.0
    step = MoistLargeStep(cfg, upload(host), upload(metrics))
    m = step.s["mass1"].clone()
    want = ko.dry_mass(host["rho"], host["ruh"], host["rvh"], metrics["rmh"], ni=24, nj=20, nk=16)
    assert abs(float(m.item()) - want) <= 1e-13 * want
    step.step()
    torch.cuda.synchronize()
    assert torch.equal(step.s["mass1"], m)
    restored = dict(host, mass1=np.array([want * 1.01], np.float64))
    again = MoistLargeStep(cfg, upload(restored), upload(metrics))
    assert float(again.s["mass1"].item()) == want * 1.01
