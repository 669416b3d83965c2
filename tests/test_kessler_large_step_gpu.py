"""The CUDA once-per-large-step Kessler transition (gm1b_kessler_large_step)
against the reference's CPU twin (golden fixtures) and against the oracle
over two consecutive transitions on a larger grid (the held rates of the
first feed the second), under the Kessler tolerances."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200 import kessler as gk
from oracle import kessler as ko
from tests.golden.make_golden import kessler_large_step_fixture
from tests.kessler_common import assert_fields_close
from tests.test_oracle_kessler_large_step import TAGS, assert_held_close, load

pytestmark = pytest.mark.gpu


def _dev(d):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in d.items()}


def _host(d):
    return {k: v.cpu().numpy() for k, v in d.items()}


def _carriers(held):
    return gk.Gm1KesslerHeldCarriers(*(held[n] for n in gk.HELD_NAMES))


@pytest.mark.parametrize("tag", TAGS)
def test_transition_matches_reference(tag):
    meta, a, held, want, want_held = load(tag)
    dev, hdev = _dev(a), _dev(held)
    t = gk.create_cuda_gm1_kessler_large_step_transition(
        dev, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dx=meta["dx"], dy=meta["dy"], dz=meta["dz"],
        dt=meta["dt"], selection=gk.Gm1KesslerDriverSelection(equation_set=meta["eqtset"]), carriers=_carriers(hdev))
    r = t.apply()
    r.ready_event.synchronize()
    got = _host(t.arrays)
    assert_fields_close(want, got)
    if meta["eqtset"] == 2:
        assert_held_close(want_held, _host(hdev), want, meta["dt"])


def test_two_transitions_match_oracle_on_a_larger_grid():
    ni, nj, nk, dz, dt = 40, 33, 30, 120.0, 10.0
    a, held = kessler_large_step_fixture(ni, nj, nk, dz, 77)
    ref_a, ref_h = {k: v.copy() for k, v in a.items()}, {k: v.copy() for k, v in held.items()}
    dev, hdev = _dev(a), _dev(held)
    t = gk.create_cuda_gm1_kessler_large_step_transition(
        dev, ni=ni, nj=nj, nk=nk, dx=500.0, dy=500.0, dz=dz, dt=dt,
        selection=gk.Gm1KesslerDriverSelection(equation_set=2), carriers=_carriers(hdev))
    for step in (1, 2):
        t.apply()
        ko.kessler_large_step(ref_a, ref_h, ni=ni, nj=nj, nk=nk, dx=500.0, dy=500.0, dz=dz, dt=dt, eqtset=2)
        torch.cuda.synchronize()
        got = _host(t.arrays)
        assert_fields_close(ref_a, got)
        assert_held_close(ref_h, _host(hdev), ref_a, dt)
    assert t.completed_transitions == 2


def test_transition_refusals():
    meta, a, held, *_ = load(TAGS[0])
    dev = _dev(a)
    t = gk.create_cuda_gm1_kessler_large_step_transition(
        dev, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], dx=1.0, dy=1.0, dz=1.0, dt=1.0,
        selection=gk.Gm1KesslerDriverSelection(equation_set=2))
    from gm1_b200.errors import CM1Refusal
    with pytest.raises(CM1Refusal):
        t.apply(final_rk=False)
    with pytest.raises(CM1Refusal):
        t.apply(pre_component_hook=lambda h: None)
