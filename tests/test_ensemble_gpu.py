"""The batched ensemble on the GPU: members of uneven sizes captured as one
CUDA graph over several streams give, after two large steps, the same words
as the same members stepped one after another with plain launches; each
member of the batch matches the same member stepped alone; and a member
steps its own state only (a member's words do not depend on its
neighbours in the batch)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.ensemble import EnsembleMember, MoistEnsemble, member_initial_state

pytestmark = pytest.mark.gpu

FIELDS = ("u3d", "v3d", "w3d", "th3d", "pp3d", "q3d", "tke3d", "rain", "ppx")
SMALL = dict(dx=1000.0, dy=1000.0, dz=300.0, dt=5.0, nsound=10)


def _members():
    return (EnsembleMember(0, 24, 20, 16, 2.0, (1000.0, -500.0), 11),
            EnsembleMember(1, 33, 27, 18, 3.0, (-2000.0, 0.0), 12),
            EnsembleMember(2, 20, 31, 16, 1.5, (0.0, 2500.0), 13))


def _words(t):
    return t.detach().cpu().numpy().view(np.uint32)


def test_batched_graph_equals_plain_one_by_one():
    members = _members()
    hosts = [member_initial_state(m, SMALL) for m in members]
    batched = MoistEnsemble(members, "cuda:0", streams=3, grid=SMALL, hosts=hosts)
    plain = MoistEnsemble(members, "cuda:0", streams=1, grid=SMALL, hosts=hosts)
    batched.step_eager()
    batched.capture()
    batched.replay()
    plain.step_eager()
    plain.step_eager()
    torch.cuda.synchronize()
    for n in range(len(members)):
        for f in FIELDS:
            assert np.array_equal(_words(batched.state(n)[f]), _words(plain.state(n)[f])), (n, f)
    batched.release()


def test_member_in_a_batch_equals_member_alone():
    members = _members()
    hosts = [member_initial_state(m, SMALL) for m in members]
    batched = MoistEnsemble(members, "cuda:0", streams=2, grid=SMALL, hosts=hosts)
    alone = MoistEnsemble(members[1:2], "cuda:0", streams=1, grid=SMALL, hosts=hosts[1:2])
    for _ in range(2):
        batched.step_eager()
        alone.step_eager()
    torch.cuda.synchronize()
    for f in FIELDS:
        assert np.array_equal(_words(batched.state(1)[f]), _words(alone.state(0)[f])), f
    # the members really differ (different sizes, bubbles and noise)
    assert batched.state(0)["th3d"].shape != batched.state(1)["th3d"].shape
    assert float(batched.state(1)["w3d"].abs().max()) > 0.0


def test_member_in_the_batch_matches_the_oracle_composition():
    """A member stepped inside the captured, multi-stream batch against the
    oracle's composition of that member alone, each field on its own scale
    (tests/moist_common.py SHORT_BARS), after 1 and 3 large steps."""
    from oracle.moist_composition import OracleMoistStep  # noqa: PLC0415
    from gm1_b200.ensemble import member_config  # noqa: PLC0415
    from tests.moist_common import SHORT_BARS, check_errors, field_errors, format_errors  # noqa: PLC0415

    members = _members()
    hosts = [member_initial_state(m, SMALL) for m in members]
    batched = MoistEnsemble(members, "cuda:0", streams=3, grid=SMALL, hosts=hosts)
    host, metrics = hosts[1]
    ref = OracleMoistStep(member_config(members[1], SMALL), {k: v.copy() for k, v in host.items()},
                          {k: v.copy() for k, v in metrics.items()})
    batched.step_eager()
    ref.step()
    torch.cuda.synchronize()
    err = field_errors(batched.state(1), ref.s)
    print("step 1", format_errors(err))
    check_errors(err, SHORT_BARS, "ensemble member 1 step 1")
    batched.capture()
    for _ in range(2):
        batched.replay()
        ref.step()
    torch.cuda.synchronize()
    err = field_errors(batched.state(1), ref.s)
    print("step 3", format_errors(err))
    check_errors(err, SHORT_BARS, "ensemble member 1 step 3")
    batched.release()
