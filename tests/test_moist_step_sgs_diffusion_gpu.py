"""The composed moist step on a stretched column with the closure's held
tendencies on (MoistStepConfig.sgs_diffusion: gettau and turbu/turbv/turbw
once per large step, added into the momentum tendencies of every RK stage,
and turbs of theta and the moisture rows into the held tendencies the
eqtset 2 composition reads; MoistStepConfig.rayleigh: CM1's upper Rayleigh
damping above zd; MoistStepConfig.dissipative_heating: CM1's idiss), on the
GPU against the oracle's composition with the same
pieces.

Bars: the first step's held momentum, theta and moisture tendencies (both
closures read the same starting words, so they differ only by the eddy
coefficients' powf/sqrtf ulps) within 1e-5 of their largest value; the
prognostic fields of the same runs are held to the binary32 oracle's own
error against the FP64 run in tests/test_moist_fp64_gpu.py (the implicit
vertical diffusion forms (solution - w)/dt, a difference of nearly equal
words, so w carries the libm ulps of the closure further than the other
fields do); the C entry point gives the Python composition's words; the
diffusion and the damping move the state; on the uniform column the damping
and the heating match too, and so does the SGS diffusion on the terrain
texts."""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest
import torch

from gm1_b200.moist_step import (SUPERCELL_STRETCHED_COLUMN, MoistLargeStep, MoistStepConfig, NativeMoistLargeStep,
                                 StretchedColumnSpec, upload, weisman_klemp_initial_state)
from oracle.moist_composition import OracleMoistStep
from tests.moist_common import check_errors, field_errors, format_errors

pytestmark = pytest.mark.gpu

SHALLOW = StretchedColumnSpec(1630.0, 40.0, 1030.0, 20.0, 200.0)
COMPARED = ("ua", "u3d", "va", "v3d", "wa", "w3d", "ppi", "pp3d", "ppx", "tha", "th3d", "qa", "q3d", "tkea", "tke3d",
            "rho", "rf", "prs", "rain", "asq", "qbudget", "kmh", "kmv", "rru", "rrv", "rrw", "mass1", "thheld", "qheld")
# u and v of the first step on their own scale (w: see the module note)
FIRST_STEP_BARS = {"u3d": (2e-5, 1e-6), "v3d": (2e-5, 1e-6)}


def _case(ni, nj, nk, column, seed, sgs_diffusion=True, rayleigh=True, dissipative_heating=None, **kw):
    idiss = sgs_diffusion and rayleigh if dissipative_heating is None else dissipative_heating
    cfg = MoistStepConfig(ni, nj, nk, 100.0, 100.0, 100.0, 0.6, 8, column=column, sgs_diffusion=sgs_diffusion,
                          rayleigh=rayleigh, dissipative_heating=idiss)
    init = dict(seed=seed, bubble_radius_m=(800.0, 400.0), bubble_center_z_m=400.0, bubble_cloud=1.0e-3,
                bubble_rain=5.0e-4)
    init.update(kw)
    host, metrics = weisman_klemp_initial_state(cfg, **init)
    return cfg, host, metrics


@pytest.mark.parametrize("sgs,rayleigh", [(True, False), (False, True), (True, True)])
def test_first_step_held_tendencies_match_the_oracle(sgs, rayleigh):
    cfg, host, metrics = _case(48, 40, 80, SUPERCELL_STRETCHED_COLUMN, 2, sgs, rayleigh,
                               bubble_radius_m=(1500.0, 1400.0), bubble_center_z_m=1500.0)
    # a wind departure from the base state in the damping layer
    host["u3d"][60:] += np.float32(2.5)
    host["v3d"][60:] -= np.float32(1.5)
    host["w3d"][60:80] += np.float32(0.25)
    for cur, base in (("ua", "u3d"), ("va", "v3d"), ("wa", "w3d")):
        host[cur][:] = host[base]
    dev = MoistLargeStep(cfg, upload(host), upload(metrics))
    ref = OracleMoistStep(cfg, {k: v.copy() for k, v in host.items()}, {k: v.copy() for k, v in metrics.items()})
    dev.step()
    ref.step()
    torch.cuda.synchronize()
    held = {n: (dev.stress[n].cpu().numpy(), ref.stress[n]) for n in ("uten", "vten", "wten")}
    held.update({n: (dev.s[n].cpu().numpy(), ref.s[n]) for n in ("thheld", "qheld")})
    for n, (g, r) in held.items():
        g, r = g.astype(np.float64), r.astype(np.float64)
        if n != "qheld" or sgs:  # the damping leaves moisture alone
            assert np.max(np.abs(r)) > 0.0, n
        assert np.max(np.abs(g - r)) <= 1e-5 * np.max(np.abs(r)), n
    err = field_errors(dev.s, ref.s)
    print("first step", format_errors(err))
    check_errors({n: err[n] for n in FIRST_STEP_BARS}, FIRST_STEP_BARS, "first step")
    dev.check()


@pytest.mark.parametrize("concurrent", [False, True])
def test_native_step_with_the_held_closure_gives_the_python_words(concurrent):
    cfg, host, metrics = _case(40, 33, 14, SHALLOW, 5)
    py = MoistLargeStep(cfg, upload(host), upload(metrics), concurrent=False)
    nat = NativeMoistLargeStep(cfg, upload(host), upload(metrics), concurrent=concurrent)
    for _ in range(2):
        py.step()
        nat.step()
    torch.cuda.synchronize()
    bad = [n for n in COMPARED
           if not np.array_equal(py.s[n].cpu().numpy().view(np.uint8), nat.s[n].cpu().numpy().view(np.uint8))]
    assert bad == []
    nat.close()


def test_the_held_closure_moves_the_state():
    cfg, host, metrics = _case(40, 33, 80, SUPERCELL_STRETCHED_COLUMN, 5, bubble_radius_m=(1500.0, 1400.0),
                               bubble_center_z_m=1500.0)
    host["u3d"][60:] += np.float32(2.5)
    host["ua"][:] = host["u3d"]
    runs = {}
    for label, c in (("off", dataclasses.replace(cfg, sgs_diffusion=False, rayleigh=False,
                                                 dissipative_heating=False)),
                     ("sgs", dataclasses.replace(cfg, rayleigh=False)),
                     ("rayleigh", dataclasses.replace(cfg, sgs_diffusion=False, dissipative_heating=False))):
        runs[label] = MoistLargeStep(c, upload(host), upload(metrics))
        runs[label].step()
    torch.cuda.synchronize()
    for n in ("u3d", "v3d", "w3d", "th3d", "q3d"):
        assert (runs["sgs"].s[n] - runs["off"].s[n]).abs().max().item() > 0.0, n
    # the damping pulls the upper-level wind back toward the base state
    du_off = (runs["off"].s["u3d"][61:81] - torch.from_numpy(host["u3d"][61:81]).cuda()).mean().item()
    du_ray = (runs["rayleigh"].s["u3d"][61:81] - torch.from_numpy(host["u3d"][61:81]).cuda()).mean().item()
    assert du_ray < du_off


def _uniform(**kw):
    cfg = MoistStepConfig(40, 33, 80, 1000.0, 1000.0, 250.0, 5.0, 10, **kw)
    host, metrics = weisman_klemp_initial_state(cfg, seed=3, bubble_radius_m=(6000.0, 1400.0), bubble_cloud=1.0e-3,
                                                bubble_rain=5.0e-4)
    # a wind departure from the base state in the damping layer (above 15 km)
    host["u3d"][64:80] += np.float32(2.5)
    host["v3d"][64:80] -= np.float32(1.5)
    host["w3d"][64:80] += np.float32(0.25)
    for cur, base in (("ua", "u3d"), ("va", "v3d"), ("wa", "w3d")):
        host[cur][:] = host[base]
    return cfg, host, metrics


@pytest.mark.parametrize("sgs", [False, True])
def test_uniform_column_held_closure_matches_the_oracle(sgs):
    """The damping and the dissipative heating do not depend on the column
    family, and the SGS stress and turbs run the terrain texts there: on
    the uniform column (configuration 2's terrain family) the first step's
    held tendencies match the oracle's and the C entry point gives the
    Python composition's words."""
    cfg, host, metrics = _uniform(sgs_diffusion=sgs, rayleigh=True, dissipative_heating=True)
    dev = MoistLargeStep(cfg, upload(host), upload(metrics))
    ref = OracleMoistStep(cfg, {k: v.copy() for k, v in host.items()}, {k: v.copy() for k, v in metrics.items()})
    nat = NativeMoistLargeStep(cfg, upload(host), upload(metrics), concurrent=True)
    dev.step()
    ref.step()
    nat.step()
    torch.cuda.synchronize()
    for n in ("uten", "vten", "wten"):
        g, r = dev.stress[n].cpu().numpy().astype(np.float64), ref.stress[n].astype(np.float64)
        assert np.max(np.abs(r)) > 0.0, n
        assert np.max(np.abs(g - r)) <= 1e-5 * np.max(np.abs(r)), n
    for n in ("thheld",) + (("qheld",) if sgs else ()):
        g, r = dev.s[n].cpu().numpy().astype(np.float64), ref.s[n].astype(np.float64)
        assert np.max(np.abs(r)) > 0.0, n
        assert np.max(np.abs(g - r)) <= 1e-5 * np.max(np.abs(r)), n
    bad = [n for n in COMPARED
           if not np.array_equal(dev.s[n].cpu().numpy().view(np.uint8), nat.s[n].cpu().numpy().view(np.uint8))]
    assert bad == []
    nat.close()
