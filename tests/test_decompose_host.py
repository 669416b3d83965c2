"""x-y decomposition by deep halos (gm1_b200/decompose.py) on the host: the
partition and the windows of every state and metric array; the two-phase
halo exchange (in-process and over two gloo ranks) leaves every halo cell of
index-coded arrays equal to the single domain's; and the oracle's composed
moist step, decomposed over 2x1 and 2x2 subdomains with a 32-cell halo and
exchanged after every large step, leaves interiors word-identical to the
single domain's after 3 steps, the stretched column also with the SGS
stress, scalar diffusion, Rayleigh damping and dissipative heating held
tendencies on (with
apmasscon off: the dry-mass correction
is a domain-wide reduction; the FP64 budgets excepted: they accumulate
per widened subdomain; a lateral-boundary history is compared on the rank
that holds that edge of the domain - elsewhere it belongs to a halo's outer
edge)."""

from __future__ import annotations

import os
import socket
from types import SimpleNamespace

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gm1_b200.decompose import HaloExchange, global_interior, interior, interior_slices, partition, window
from gm1_b200.restart import CARRIED
from oracle.moist_composition import OracleMoistStep
from oracle.moist_initial import moist_state_shapes, weisman_klemp_initial_state

HALO = 32
COMPARED = tuple(n for n in CARRIED if n not in ("asq", "qbudget"))
# a lateral-boundary history belongs to the rank on that edge of the domain
EDGE = {"radbcw": lambda s, px, py: s.px == 0, "radbce": lambda s, px, py: s.px == px - 1,
        "radbcs": lambda s, px, py: s.py == 0, "radbcn": lambda s, px, py: s.py == py - 1}


def compared(s, px, py):
    return tuple(n for n in COMPARED if n not in EDGE or EDGE[n](s, px, py))


def _cfg(ni, nj, stretched=False, sgs_diffusion=False):
    column = SimpleNamespace(ztop_m=20800.0, str_bot_m=200.0, str_top_m=15800.0, dz_bot_m=20.0,
                             dz_top_m=500.0) if stretched else None
    nk, dx, dz, dt, ns = (80, 100.0, 100.0, 0.6, 8) if stretched else (12, 1000.0, 250.0, 5.0, 10)
    # the dry-mass correction is a domain-wide reduction: off in a decomposed run
    return SimpleNamespace(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, dt=dt, nsound=ns, alph=0.60, kdiv=0.10,
                           lateral_sides=(2, 2, 2, 2), obc=0x2222, column=column, apmasscon=False,
                           sgs_diffusion=sgs_diffusion, rayleigh=sgs_diffusion,
                           dissipative_heating=sgs_diffusion)


def _start(cfg):
    return weisman_klemp_initial_state(cfg, seed=5, bubble_radius_m=(12 * cfg.dx, 5 * cfg.dz),
                                       bubble_center_z_m=5 * cfg.dz, bubble_cloud=1.0e-3, bubble_rain=5.0e-4)


def _coded(ni, nj, nk):
    """Every state array filled with distinct words (its global index)."""
    out = {}
    for q, (n, sh) in enumerate(moist_state_shapes(ni, nj, nk).items()):
        out[n] = (np.arange(int(np.prod(sh)), dtype=np.float64).reshape(sh) + 1.0e6 * q).astype(np.float32)
    return out


def test_partition_and_windows():
    subs = partition(100, 70, 2, 2, 16)
    assert [(s.x0, s.nx, s.y0, s.ny) for s in subs] == [(0, 50, 0, 35), (50, 50, 0, 35), (0, 50, 35, 35),
                                                        (50, 50, 35, 35)]
    assert [(s.hw, s.he, s.hs, s.hn) for s in subs] == [(0, 16, 0, 16), (16, 0, 0, 16), (0, 16, 16, 0),
                                                        (16, 0, 16, 0)]
    with pytest.raises(ValueError, match="narrower"):
        partition(40, 10, 2, 1, 32)
    g = _coded(100, 70, 4)
    s = subs[3]
    w = window(g, 100, 70, s)
    assert w["u3d"].shape == (6, s.enj + 6, s.eni + 7) and w["v3d"].shape == (6, s.enj + 7, s.eni + 6)
    assert w["pp3d"].shape == (6, s.enj + 2, s.eni + 2) and w["radbcs"].shape == (6, s.eni + 6)
    assert w["radbcw"].shape == (6, s.enj + 6) and w["uh"].shape == (s.eni + 6,) and w["th0"].shape == (4,)
    # the window's interior is the global interior
    for n in ("u3d", "v3d", "w3d", "pp3d", "th3d", "q3d", "rain", "radbcs", "radbcw", "uh", "rvh"):
        assert np.array_equal(interior(w, s, [n])[n], global_interior(g, 100, 70, s, [n])[n]), n


@pytest.mark.parametrize("px,py", [(2, 1), (1, 2), (2, 2), (3, 2)])
def test_in_process_exchange_fills_every_facing_halo(px, py):
    ni, nj, nk = 90, 80, 3
    g = _coded(ni, nj, nk)
    subs = partition(ni, nj, px, py, 12)
    local, tensors = {}, {}
    for s in subs:
        w = window(g, ni, nj, s)
        for n in CARRIED:  # every halo word scrambled, the interior kept
            keep = w[n][interior_slices(n, w[n].shape, s)].copy()
            w[n][...] = -7.0
            w[n][interior_slices(n, w[n].shape, s)] = keep
        local[s.rank] = w
        tensors[s.rank] = {n: torch.from_numpy(w[n]) for n in CARRIED}
    HaloExchange(subs, tensors).exchange()
    for s in subs:
        got, want = local[s.rank], window(g, ni, nj, s)
        for n in CARRIED:
            # the interior and every halo that faces a rank hold the single
            # domain's words; only the outer ghosts of the widened block may not
            sl = interior_slices(n, got[n].shape, _widened(s))
            assert np.array_equal(got[n][sl], want[n][sl]), (s.rank, n)
            assert np.array_equal(got[n][interior_slices(n, got[n].shape, s)],
                                  global_interior(g, ni, nj, s, [n])[n]), (s.rank, n)


def _widened(s):
    """The subdomain seen as one block of its widened cells (halo included)."""
    return type(s)(s.rank, s.px, s.py, s.ex0, s.eni, s.ey0, s.enj, 0, 0, 0, 0)


def _decomposed_oracle(cfg, host, metrics, subs, steps):
    ni, nj = cfg.ni, cfg.nj
    runs, tensors = {}, {}
    for s in subs:
        c = SimpleNamespace(**{**vars(cfg), "ni": s.eni, "nj": s.enj})
        st, mt = window(host, ni, nj, s), window(metrics, ni, nj, s)
        runs[s.rank] = OracleMoistStep(c, st, mt)
        tensors[s.rank] = {n: torch.from_numpy(st[n]) for n in CARRIED}
    x = HaloExchange(subs, tensors)
    for _ in range(steps):
        for r in runs.values():
            r.step()
        x.exchange()
    return runs


@pytest.mark.parametrize("px,py,stretched,stress", [(2, 1, False, False), (2, 2, False, False), (2, 1, True, False),
                                                    (1, 2, True, True)])
def test_decomposed_oracle_composition_is_the_single_domain(px, py, stretched, stress):
    cfg = _cfg(80 if px > 1 else 40, 72 if py > 1 else 24, stretched, stress)
    host, metrics = _start(cfg)
    single = OracleMoistStep(cfg, {k: v.copy() for k, v in host.items()}, {k: v.copy() for k, v in metrics.items()})
    subs = partition(cfg.ni, cfg.nj, px, py, HALO)
    runs = _decomposed_oracle(cfg, host, metrics, subs, 3)
    for _ in range(3):
        single.step()
    for s in subs:
        names = compared(s, px, py)
        got = interior(runs[s.rank].s, s, names)
        want = global_interior(single.s, cfg.ni, cfg.nj, s, names)
        bad = [n for n in names if not np.array_equal(got[n].view(np.uint8), want[n].view(np.uint8))]
        assert not bad, (s.rank, bad)
    assert float(single.s["q3d"][2].max()) > 0.0


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg = _cfg(80, 24)
        host, metrics = _start(cfg)
        subs = partition(cfg.ni, cfg.nj, 2, 1, HALO)
        s = subs[rank]
        c = SimpleNamespace(**{**vars(cfg), "ni": s.eni, "nj": s.enj})
        st, mt = window(host, cfg.ni, cfg.nj, s), window(metrics, cfg.ni, cfg.nj, s)
        run = OracleMoistStep(c, st, mt)
        x = HaloExchange(subs, {rank: {n: torch.from_numpy(st[n]) for n in CARRIED}})
        for _ in range(3):
            run.step()
            x.exchange()
        out.put((rank, interior(run.s, s, COMPARED)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_step_the_single_domain():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cfg = _cfg(80, 24)
    host, metrics = _start(cfg)
    single = OracleMoistStep(cfg, host, metrics)
    for _ in range(3):
        single.step()
    for s in partition(cfg.ni, cfg.nj, 2, 1, HALO):
        names = compared(s, 2, 1)
        want = global_interior(single.s, cfg.ni, cfg.nj, s, names)
        bad = [n for n in names if not np.array_equal(results[s.rank][n].view(np.uint8), want[n].view(np.uint8))]
        assert not bad, (s.rank, bad)
