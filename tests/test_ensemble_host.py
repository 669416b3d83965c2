"""Host logic of the batched ensemble and of multi-rank runs, on CPU:
member draws (seeded, in range, reproducible), the member shard over ranks
(every member on exactly one rank, balanced by cells), and the rank
reductions of the job timing on a two-process gloo group."""

from __future__ import annotations

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from gm1_b200.ensemble import ENSEMBLE_SEED, ensemble_members
from gm1_b200.replicas import job_rate, max_over_ranks, member_shard, sum_over_ranks


def test_members_are_seeded_and_in_range():
    a = ensemble_members(64)
    b = ensemble_members(64, seed=ENSEMBLE_SEED)
    assert a == b
    assert [m.index for m in a] == list(range(64))
    for m in a:
        assert 48 <= m.ni <= 160 and 48 <= m.nj <= 160 and 40 <= m.nk <= 64
        assert 1.0 <= m.bubble_k <= 3.0
        assert all(abs(o) <= 5000.0 for o in m.offset_m)
        assert m.seed == ENSEMBLE_SEED * 1000 + m.index
    assert len({(m.ni, m.nj, m.nk) for m in a}) > 32  # uneven sizes
    assert ensemble_members(64, seed=6) != a
    total = sum(m.cells for m in a)
    assert 20_000_000 < total < 60_000_000  # about 36 M cells at the means


def test_member_draws_refuse_bad_arguments():
    with pytest.raises(ValueError):
        ensemble_members(0)
    with pytest.raises(ValueError):
        ensemble_members(4, nx=(4, 10))


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_member_shard_covers_every_member_once_and_balances_cells(world):
    cells = [m.cells for m in ensemble_members(64)]
    shards = [member_shard(cells, r, world) for r in range(world)]
    flat = sorted(m for s in shards for m in s)
    assert flat == list(range(64))
    loads = [sum(cells[m] for m in s) for s in shards]
    assert max(loads) - min(loads) <= max(cells)


def test_member_shard_refuses_bad_ranks():
    with pytest.raises(ValueError):
        member_shard([1, 2], 2, 2)
    with pytest.raises(ValueError):
        member_shard([1, 2], 0, 0)
    with pytest.raises(ValueError):
        member_shard([1, -2], 0, 1)


def test_reductions_without_a_group_return_the_local_value():
    assert max_over_ranks(3.5) == 3.5
    assert sum_over_ranks(2.0) == 2.0
    assert job_rate(10.0, 2.0) == (10.0, 2.0, 5.0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cells = [m.cells for m in ensemble_members(64)]
        mine = member_shard(cells, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        units = float(sum(cells[m] for m in mine))
        seconds = 1.0 + rank  # rank r pretends its timed region took 1 + r s
        total, worst, rate = job_rate(units, seconds)
        out.put((rank, gathered, total, worst, rate, max_over_ranks(float(rank * 10))))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_members_and_reduce_the_timing():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cells = [m.cells for m in ensemble_members(64)]
    for rank, gathered, total, worst, rate, mx in results:
        assert sorted(m for s in gathered for m in s) == list(range(64))
        assert not set(gathered[0]) & set(gathered[1])
        assert gathered[rank] == member_shard(cells, rank, world)
        assert total == float(sum(cells))
        assert worst == 2.0  # the slower rank's seconds
        assert rate == total / 2.0
        assert mx == 10.0
