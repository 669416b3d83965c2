"""Batched ensembles of uneven moist domains on one GPU.

Each member is a whole Weisman-Klemp supercell domain of its own size, with
its own warm bubble, stepped by the composed moist large step
(:class:`gm1_b200.moist_step.MoistLargeStep`).  Two ways to run a set of
members:

* batched (:meth:`MoistEnsemble.capture` + :meth:`MoistEnsemble.replay`):
  the members' steps are spread over a few CUDA streams forked from one
  capture stream and joined back, and the whole ensemble step is captured
  once as a single CUDA graph, so small members overlap on the SMs and the
  host issues one graph launch per step;
* plain (:meth:`MoistEnsemble.step_eager` with one stream): the members one
  after another with ordinary launches, the way a caller without batching
  steps them.

Both run the same kernels on the same words, so they produce the same state
bit for bit.  Members draw their sizes and bubbles from a seeded generator
(:func:`ensemble_members`): nx, ny uniform on 48..160, nz on 40..64, bubble
amplitude U[1, 3] K, bubble centre jittered U(+-5 km) in x and y.
"""

from __future__ import annotations

from collections.abc import Sequence
from dataclasses import dataclass
from typing import Any

import numpy as np
import torch

from .moist_step import MoistLargeStep, MoistStepConfig, upload, weisman_klemp_initial_state

ENSEMBLE_SEED = 5
# dx = dy = 1 km; dz = 300 m puts the lid at 12-19 km for nz 40..64
ENSEMBLE_GRID = dict(dx=1000.0, dy=1000.0, dz=300.0, dt=5.0, nsound=10)


@dataclass(frozen=True)
class EnsembleMember:
    index: int
    ni: int
    nj: int
    nk: int
    bubble_k: float
    offset_m: tuple[float, float]
    seed: int

    @property
    def cells(self) -> int:
        return self.ni * self.nj * self.nk


def ensemble_members(count: int = 64, *, seed: int = ENSEMBLE_SEED, nx: tuple[int, int] = (48, 160),
                     nz: tuple[int, int] = (40, 64), bubble_k: tuple[float, float] = (1.0, 3.0),
                     jitter_m: float = 5000.0) -> tuple[EnsembleMember, ...]:
    """``count`` members drawn from ``numpy.random.default_rng(seed)`` in
    member order: ni, nj, nk (inclusive bounds), the bubble amplitude, then
    the x and y centre offsets; member m's noise seed is ``seed * 1000 + m``."""
    if count < 1:
        raise ValueError("an ensemble needs at least one member")
    if not (5 <= nx[0] <= nx[1] and 4 <= nz[0] <= nz[1]):
        raise ValueError("member sizes must be at least 5 columns and 4 levels")
    rng = np.random.default_rng(seed)
    out = []
    for m in range(count):
        ni = int(rng.integers(nx[0], nx[1] + 1))
        nj = int(rng.integers(nx[0], nx[1] + 1))
        nk = int(rng.integers(nz[0], nz[1] + 1))
        amp = float(rng.uniform(bubble_k[0], bubble_k[1]))
        ox, oy = (float(v) for v in rng.uniform(-jitter_m, jitter_m, 2))
        out.append(EnsembleMember(m, ni, nj, nk, amp, (ox, oy), seed * 1000 + m))
    return tuple(out)


def member_config(member: EnsembleMember, grid: dict | None = None) -> MoistStepConfig:
    g = dict(ENSEMBLE_GRID if grid is None else grid)
    return MoistStepConfig(member.ni, member.nj, member.nk, g["dx"], g["dy"], g["dz"], g["dt"], g["nsound"])


def member_initial_state(member: EnsembleMember, grid: dict | None = None) -> tuple[dict, dict]:
    """Host state and metrics of one member: the Weisman-Klemp start with the
    member's bubble (radius 10 km x 1.5 km at 1.5 km) and U(+-0.1 K) noise."""
    cfg = member_config(member, grid)
    return weisman_klemp_initial_state(cfg, seed=member.seed, bubble_k=member.bubble_k, noise_k=0.1,
                                       bubble_radius_m=(10000.0, 1500.0), bubble_center_z_m=1500.0,
                                       bubble_offset_m=member.offset_m)


class MoistEnsemble:
    """The members of ``members`` resident on ``device``, each with its own
    state and a :class:`MoistLargeStep` on one of ``streams`` CUDA streams
    (member m on stream m mod streams).  ``hosts`` (the members' host states
    and metrics, in member order) may be passed to skip building them."""

    def __init__(self, members: Sequence[EnsembleMember], device: torch.device | str, *, streams: int = 8,
                 grid: dict | None = None, hosts: Sequence[tuple[dict, dict]] | None = None,
                 tuner: Any | None = None) -> None:
        if not members:
            raise ValueError("an ensemble needs at least one member")
        if streams < 1:
            raise ValueError("streams must be >= 1")
        self.device = torch.device(device)
        self.members = tuple(members)
        self.main = torch.cuda.Stream(self.device)
        self.streams = [self.main] if streams == 1 else [torch.cuda.Stream(self.device)
                                                          for _ in range(min(streams, len(members)))]
        self.steps: list[MoistLargeStep] = []
        for n, mb in enumerate(self.members):
            host, metrics = member_initial_state(mb, grid) if hosts is None else hosts[n]
            st = self.streams[n % len(self.streams)]
            with torch.cuda.stream(st):
                # members already overlap one another, so each steps its own
                # operations in order on its stream
                # with a tuner (gm1_b200.autotune.Autotuner) each member's
                # advection z-chunk is picked for its grid shape, once per
                # shape: members of one shape share the table's entry
                self.steps.append(MoistLargeStep(member_config(mb, grid), upload(host, self.device),
                                                 upload(metrics, self.device), stream=st, concurrent=False,
                                                 tuner=tuner))
        self.graph: torch.cuda.CUDAGraph | None = None

    @property
    def cells(self) -> int:
        return sum(m.cells for m in self.members)

    def _fork_join(self) -> None:
        if len(self.streams) == 1:
            for s in self.steps:
                s.step()
            return
        fork = torch.cuda.Event()
        fork.record(self.main)
        for st in self.streams:
            st.wait_event(fork)
        for s in self.steps:
            s.step()
        for st in self.streams:
            done = torch.cuda.Event()
            done.record(st)
            self.main.wait_event(done)

    def step_eager(self) -> None:
        """One large step of every member with ordinary launches, ordered
        after the work already on the main stream and before what follows."""
        with torch.cuda.stream(self.main):
            self._fork_join()

    def capture(self) -> None:
        """Capture one large step of every member as one CUDA graph (run
        :meth:`step_eager` once first so every lazily created resource exists)."""
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.main):
            self._fork_join()
        self.graph = g

    def replay(self) -> None:
        """One large step of every member: the captured graph, launched on the
        main stream."""
        if self.graph is None:
            raise RuntimeError("capture() the ensemble step before replaying it")
        with torch.cuda.stream(self.main):
            self.graph.replay()

    def release(self) -> None:
        self.graph = None

    def state(self, index: int) -> dict[str, Any]:
        return self.steps[index].s
