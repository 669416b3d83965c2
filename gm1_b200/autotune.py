"""Per-grid-shape launch tuning.

The tiled stencil kernels march a z-chunk of levels per CTA over a fixed
x-y tile; how many levels one CTA should march depends on the grid: a large
plane has tiles enough to fill the 148 SMs with long chunks (fewer halo
re-reads per level), a small plane needs short chunks to have CTAs enough at
all.  ``Autotuner`` times each candidate once per (kernel, grid shape) with
CUDA events on the launching stream and keeps the fastest; the table can be
saved to and loaded from a JSON file so that a production run pays the
search once.
"""

from __future__ import annotations

import json
from pathlib import Path
from typing import Callable, Iterable

import torch

LEVEL_CHUNKS = (1, 2, 4, 8, 16)


class Autotuner:
    def __init__(self, path: str | Path | None = None, *, warmup: int = 2, repeats: int = 5):
        self.path = None if path is None else Path(path)
        self.warmup, self.repeats = warmup, repeats
        self.table: dict[str, dict] = {}
        if self.path is not None and self.path.exists():
            self.table = json.loads(self.path.read_text())

    @staticmethod
    def key(kind: str, ni: int, nj: int, nk: int) -> str:
        return f"{kind}:{ni}x{nj}x{nk}"

    def choose(self, kind: str, ni: int, nj: int, nk: int, run: Callable[[int], None],
               candidates: Iterable[int] = LEVEL_CHUNKS) -> int:
        """The fastest candidate for ``run(candidate)`` (one launch of the
        kernel with that setting on the current stream); cached per key."""
        k = self.key(kind, ni, nj, nk)
        if k in self.table:
            return int(self.table[k]["best"])
        stream = torch.cuda.current_stream()
        times = {}
        for c in candidates:
            if c > nk:
                continue
            for _ in range(self.warmup):
                run(c)
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            for _ in range(self.repeats):
                run(c)
            end.record(stream)
            end.synchronize()
            times[c] = start.elapsed_time(end) / self.repeats
        best = min(times, key=times.get)
        self.table[k] = {"best": best, "ms": {str(c): t for c, t in times.items()}}
        return best

    def save(self) -> None:
        if self.path is not None:
            self.path.write_text(json.dumps(self.table, indent=1, sort_keys=True))


_default: Autotuner | None = None


def default_tuner() -> Autotuner:
    global _default
    if _default is None:
        _default = Autotuner()
    return _default
