"""Host-side rank logic of multi-GPU runs: one process per GPU, each rank
owning whole domains, and no collective on the data path.

A single moist domain does not shard in this build (its x-y halo exchange
is not built), so N ranks run N independent replicas of it.  An ensemble
shards by member: each rank steps the members assigned to it, the members
balanced by cell count.  The only collectives are the scalar reductions of
the job's timing (max over ranks) and of the units processed (sum over
ranks), on whatever backend the process group uses (NCCL on the GPUs, gloo
in the CPU tests).
"""

from __future__ import annotations

from collections.abc import Sequence

import torch
import torch.distributed as dist


def member_shard(cells: Sequence[int], rank: int, world: int) -> list[int]:
    """Indices of the members rank ``rank`` of ``world`` steps: longest
    processing time first (members by cell count, largest first, ties by
    index), each to the rank with the fewest cells so far (ties to the lowest
    rank).  Every member lands on exactly one rank; the result is sorted."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} is not in a world of {world}")
    if any(int(c) < 0 for c in cells):
        raise ValueError("member cell counts must be >= 0")
    load = [0] * world
    owner = [0] * len(cells)
    for m in sorted(range(len(cells)), key=lambda q: (-int(cells[q]), q)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[m] = r
        load[r] += int(cells[m])
    return [m for m in range(len(cells)) if owner[m] == rank]


def _reduce(x: float, op, device: torch.device | None) -> float:
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or torch.device("cpu"))
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x: float, device: torch.device | None = None) -> float:
    """The largest x over the ranks of the default group (x itself without
    one).  Every rank must call it at the same point."""
    return _reduce(x, dist.ReduceOp.MAX, device)


def sum_over_ranks(x: float, device: torch.device | None = None) -> float:
    """The sum of x over the ranks of the default group."""
    return _reduce(x, dist.ReduceOp.SUM, device)


def job_rate(units: float, seconds: float, device: torch.device | None = None) -> tuple[float, float, float]:
    """(units of all ranks, the slowest rank's seconds, units/s of the whole
    job) for units processed by this rank in its own timed seconds."""
    total = sum_over_ranks(units, device)
    worst = max_over_ranks(seconds, device)
    return total, worst, total / worst if worst > 0 else float("inf")
