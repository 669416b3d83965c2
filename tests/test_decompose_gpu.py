"""x-y decomposition by deep halos on the GPU: the composed moist step of
one domain run as 2x1 and 2x2 widened subdomains (32-cell halos) held by
one process on one device, with the halo strips of the carried arrays
exchanged by device copies after every large step, leaves interiors that are
the single-domain GPU step's words after 3 steps: the Python composition on
the uniform and the stretched column with the dry-air mass correction (its
ledger added over the subdomains; the binary64 mass1 within 1e-13 of the
single domain's, summed in another order) and without it, and the C entry
point (one call per step, so the correction off) on the 80-level stretched
column.  The FP64 budgets accumulate per widened subdomain; a
lateral-boundary history is compared on the rank that holds that edge of the
domain."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200.decompose import DecomposedRun, HaloExchange, global_interior, interior, local_steps, partition
from gm1_b200.moist_step import (SUPERCELL_STRETCHED_COLUMN, MoistLargeStep, MoistStepConfig, NativeMoistLargeStep,
                                 upload, weisman_klemp_initial_state)
from gm1_b200.restart import CARRIED

pytestmark = pytest.mark.gpu

HALO = 32
EDGE = {"radbcw": lambda s, px, py: s.px == 0, "radbce": lambda s, px, py: s.px == px - 1,
        "radbcs": lambda s, px, py: s.py == 0, "radbcn": lambda s, px, py: s.py == py - 1}
COMPARED = tuple(n for n in CARRIED if n not in ("asq", "qbudget", "mass1"))

CASES = {
    "python-uniform-2x1": (MoistLargeStep, MoistStepConfig(96, 40, 16, 1000.0, 1000.0, 250.0, 5.0, 10,
                                                           apmasscon=False), 2, 1),
    "python-uniform-2x2": (MoistLargeStep, MoistStepConfig(80, 72, 16, 1000.0, 1000.0, 250.0, 5.0, 10,
                                                           apmasscon=False), 2, 2),
    "native-stretched-2x1": (NativeMoistLargeStep, MoistStepConfig(80, 32, 80, 100.0, 100.0, 100.0, 0.6, 8,
                                                                   column=SUPERCELL_STRETCHED_COLUMN,
                                                                   apmasscon=False), 2, 1),
    # the dry-air mass correction on: its ledger added over the subdomains
    "python-apmasscon-2x1": (MoistLargeStep, MoistStepConfig(96, 40, 16, 1000.0, 1000.0, 250.0, 5.0, 10), 2, 1),
    "python-apmasscon-2x2": (MoistLargeStep, MoistStepConfig(80, 72, 16, 1000.0, 1000.0, 250.0, 5.0, 10), 2, 2),
    "python-apmasscon-stretched-2x1": (MoistLargeStep, MoistStepConfig(80, 32, 80, 100.0, 100.0, 100.0, 0.6, 8,
                                                                       column=SUPERCELL_STRETCHED_COLUMN), 2, 1),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_decomposed_step_is_the_single_domain(case):
    kind, cfg, px, py = CASES[case]
    host, metrics = weisman_klemp_initial_state(cfg, seed=5, bubble_radius_m=(12 * cfg.dx, 1400.0),
                                                bubble_center_z_m=1400.0, bubble_cloud=1.0e-3, bubble_rain=5.0e-4)
    single = kind(cfg, upload(host), upload(metrics))
    subs = partition(cfg.ni, cfg.nj, px, py, HALO)
    steps = local_steps(cfg, host, metrics, subs, range(len(subs)),
                        lambda c, st, mt: kind(c, upload(st), upload(mt)))
    run = DecomposedRun(steps, HaloExchange(subs, {r: steps[r].s for r in steps}))
    for _ in range(3):
        single.step()
        run.step()
    torch.cuda.synchronize()
    for s in subs:
        names = tuple(n for n in COMPARED if n not in EDGE or EDGE[n](s, px, py))
        got = interior(steps[s.rank].s, s, names)
        want = global_interior(single.s, cfg.ni, cfg.nj, s, names)
        bad = [n for n in names if not np.array_equal(got[n].view(np.uint8), want[n].view(np.uint8))]
        assert not bad, (case, s.rank, bad)
        if cfg.apmasscon:  # the domain's ledger, summed in another order
            m1, m0 = float(steps[s.rank].s["mass1"].item()), float(single.s["mass1"].item())
            assert abs(m1 - m0) <= 1e-13 * m0, (case, m1, m0)
