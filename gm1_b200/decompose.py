"""x-y domain decomposition of one moist domain over ranks, by deep halos.

The plain method shards a single domain by 2-D x-y decomposition.  This
build does it without touching a kernel: each rank steps its subdomain
widened by a halo of `halo` cells on every side that faces another rank,
as an ordinary open-sided domain, and after every large step the ranks
exchange the halo strips of the arrays the step carries from one large step
to the next (the restart inventory, gm1_b200/restart.py CARRIED).  A large
step moves information at most a bounded number of cells (fifth-order
advection: 3 cells per RK stage; the acoustic substeps: 1 cell per small
step; the closure and the fills: a few), so with the halo wider than that
bound every interior cell of every rank sees exactly the words the single
domain would, and the interiors are the single domain's step word for word
(tests/test_decompose_host.py on gloo ranks, tests/test_decompose_gpu.py on
the GPU).  The strips of a halo that faces a rank are overwritten before the
next step reads them; the outer ghost cells of a halo are scratch of the fake
edge.  Exchanges run in two phases, x then y over the x-widened rows, so the
corner halos come from the diagonal neighbour through the x neighbour's
fresh strip.  The FP64 Kessler budgets (asq, qbudget) accumulate over each
rank's widened subdomain and are not reduced here.  The final-RK dry-air
mass correction, a domain-wide reduction, is formed from the level sums of
every subdomain's own cells added over the subdomains (DecomposedRun).

The exchange (one message per neighbour per phase, packed contiguous) runs
over torch.distributed point-to-point sends (gloo on CPU tensors, NCCL on
CUDA tensors over NVLink) or, for several subdomains held by one process,
as device copies.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Callable, Iterable, Mapping

import numpy as np

from .restart import CARRIED

# 1-D arrays along x / along y; 2-D lateral-boundary arrays with a single
# horizontal axis (last): the W/E histories run along y, the S/N along x
X1D = frozenset({"uh", "ruf", "ruh"})
Y1D = frozenset({"vh", "rvf", "rvh"})
YLINE = frozenset({"radbcw", "radbce"})
XLINE = frozenset({"radbcs", "radbcn"})
# low-side ghost cells of an axis of extent n + extra (padded lane ng = 3,
# pressure lane 1, compact and face arrays 0)
_GHOSTS = {0: 0, 1: 0, 2: 1, 6: 3, 7: 3}


@dataclass(frozen=True)
class Subdomain:
    """One rank's share: interior cells [x0, x0+nx) x [y0, y0+ny) of the
    global grid, widened by hw/he/hs/hn halo cells (0 on a global edge)."""

    rank: int
    px: int
    py: int
    x0: int
    nx: int
    y0: int
    ny: int
    hw: int
    he: int
    hs: int
    hn: int

    @property
    def ex0(self) -> int:
        return self.x0 - self.hw

    @property
    def ey0(self) -> int:
        return self.y0 - self.hs

    @property
    def eni(self) -> int:
        return self.nx + self.hw + self.he

    @property
    def enj(self) -> int:
        return self.ny + self.hs + self.hn


def _split(n: int, parts: int) -> list[tuple[int, int]]:
    base, rem = divmod(n, parts)
    out, s = [], 0
    for p in range(parts):
        w = base + (1 if p < rem else 0)
        out.append((s, w))
        s += w
    return out


def partition(ni: int, nj: int, px: int, py: int, halo: int) -> list[Subdomain]:
    """Ranks px*py in row-major order (rank = qy*px + qx); every interior at
    least `halo` cells wide in a split direction, so a halo lies inside one
    neighbour's interior."""
    if px < 1 or py < 1 or halo < 1:
        raise ValueError("px, py and halo must be >= 1")
    xs, ys = _split(ni, px), _split(nj, py)
    if (px > 1 and min(w for _, w in xs) < halo) or (py > 1 and min(w for _, w in ys) < halo):
        raise ValueError(f"a {ni}x{nj} grid over {px}x{py} ranks leaves an interior narrower than the {halo}-cell halo")
    subs = []
    for qy, (y0, ny) in enumerate(ys):
        for qx, (x0, nx) in enumerate(xs):
            subs.append(Subdomain(qy * px + qx, qx, qy, x0, nx, y0, ny, halo if qx > 0 else 0,
                                  halo if qx < px - 1 else 0, halo if qy > 0 else 0, halo if qy < py - 1 else 0))
    return subs


def _axes(name: str, shape: tuple[int, ...], ni: int, nj: int) -> tuple[int | None, int | None]:
    """(x axis, y axis) of an array of the state or the metrics."""
    if len(shape) == 1:
        return (0, None) if name in X1D else ((None, 0) if name in Y1D else (None, None))
    if name in YLINE:
        return None, len(shape) - 1
    if name in XLINE:
        return len(shape) - 1, None
    xa, ya = len(shape) - 1, len(shape) - 2
    ok = shape[xa] - ni in _GHOSTS and shape[ya] - nj in _GHOSTS
    return (xa, ya) if ok else (None, None)


def window(arrays: Mapping[str, np.ndarray], ni: int, nj: int, sub: Subdomain) -> dict[str, np.ndarray]:
    """The widened subdomain's copy of global host arrays (state or metrics):
    every x/y axis cut to the subdomain's cells plus the axis's own ghost
    layout."""
    out = {}
    for n, a in arrays.items():
        a = np.asarray(a)
        xa, ya = _axes(n, a.shape, ni, nj)
        sl = [slice(None)] * a.ndim
        if xa is not None:
            e = a.shape[xa] - ni
            sl[xa] = slice(sub.ex0, sub.ex0 + sub.eni + e)
        if ya is not None:
            e = a.shape[ya] - nj
            sl[ya] = slice(sub.ey0, sub.ey0 + sub.enj + e)
        out[n] = np.array(a[tuple(sl)], order="C", copy=True)
    return out


@dataclass(frozen=True)
class Transfer:
    """Cells [c0, c1) along `axis_kind` ('x' or 'y') of global coordinates,
    sent from rank src (from its interior) into rank dst's halo."""

    src: int
    dst: int
    axis_kind: str
    c0: int
    c1: int


def _transfers(subs: list[Subdomain], phase: str) -> list[Transfer]:
    by = {(s.px, s.py): s for s in subs}
    out = []
    for s in subs:
        if phase == "x":
            for dq, lo, hi in ((-1, s.x0 - s.hw, s.x0), (1, s.x0 + s.nx, s.x0 + s.nx + s.he)):
                nb = by.get((s.px + dq, s.py))
                if nb is not None and hi > lo:
                    out.append(Transfer(nb.rank, s.rank, "x", lo, hi))
        else:
            for dq, lo, hi in ((-1, s.y0 - s.hs, s.y0), (1, s.y0 + s.ny, s.y0 + s.ny + s.hn)):
                nb = by.get((s.px, s.py + dq))
                if nb is not None and hi > lo:
                    out.append(Transfer(nb.rank, s.rank, "y", lo, hi))
    return out


def _slices(name: str, shape, sub: Subdomain, t: Transfer) -> tuple[slice, ...] | None:
    """Index slices of cells [t.c0, t.c1) in `sub`'s widened array (the
    other horizontal axis whole: in phase y that includes the x halos)."""
    xa, ya = _axes(name, shape, sub.eni, sub.enj)
    axis, origin, n = (xa, sub.ex0, sub.eni) if t.axis_kind == "x" else (ya, sub.ey0, sub.enj)
    if axis is None:
        return None
    off = _GHOSTS[shape[axis] - n]
    sl = [slice(None)] * len(shape)
    sl[axis] = slice(t.c0 - origin + off, t.c1 - origin + off)
    return tuple(sl)


class HaloExchange:
    """The halo strips of `names` between the subdomains of `subs`, after
    every large step (`exchange`).  `local` holds {rank: state dict of
    tensors} for the subdomains this process steps; with torch.distributed
    initialised, strips to and from other processes travel as one packed
    message per neighbour per phase."""

    def __init__(self, subs: list[Subdomain], local: Mapping[int, Mapping[str, Any]], names: Iterable[str] = CARRIED,
                 group: Any = None) -> None:
        self.subs = {s.rank: s for s in subs}
        self.local = dict(local)
        self.names = tuple(names)
        self.group = group
        self.phases = [_transfers(subs, "x"), _transfers(subs, "y")]

    def _views(self, rank: int, t: Transfer, as_src: bool):
        st, sub = self.local[rank], self.subs[rank]
        out = []
        for n in self.names:
            a = st[n]
            sl = _slices(n, tuple(a.shape), sub, t)
            if sl is not None:
                out.append(a[sl])
        return out

    def exchange(self) -> None:
        import torch  # noqa: PLC0415
        import torch.distributed as dist  # noqa: PLC0415

        for transfers in self.phases:
            sends, recvs, unpack = [], [], []
            for t in transfers:
                src_here, dst_here = t.src in self.local, t.dst in self.local
                if src_here and dst_here:
                    for d, s in zip(self._views(t.dst, t, False), self._views(t.src, t, True)):
                        d.copy_(s)
                elif src_here:
                    parts = [v.reshape(-1) for v in self._views(t.src, t, True)]
                    buf = torch.cat(parts)
                    sends.append(dist.P2POp(dist.isend, buf, t.dst, self.group))
                elif dst_here:
                    views = self._views(t.dst, t, False)
                    buf = torch.empty(sum(v.numel() for v in views), dtype=views[0].dtype, device=views[0].device)
                    recvs.append(dist.P2POp(dist.irecv, buf, t.src, self.group))
                    unpack.append((buf, views))
            ops = sends + recvs
            if ops:
                for req in dist.batch_isend_irecv(ops):
                    req.wait()
            for buf, views in unpack:
                q = 0
                for v in views:
                    v.copy_(buf[q:q + v.numel()].view(v.shape))
                    q += v.numel()


class DecomposedRun:
    """Large steps of a decomposed domain: each local subdomain's step
    (an object with .step(), e.g. MoistLargeStep on the widened
    subdomain's state) followed by the halo exchange.

    With the final-RK dry-air mass correction on (the steps' cfg.apmasscon),
    the correction is the domain's: each step runs up to the ledger
    (step_begin), the level partials of every subdomain's own cells are added
    - the local subdomains' in rank order, then over processes by an
    all-reduce - and every subdomain finishes from the same sums
    (step_end).  The ledger mass1 of the starting state is formed the same
    way at set-up.  The added binary64 ledgers differ from the single
    domain's only in the order of their sums, so the binary32 correction is
    the single domain's word unless its binary64 value lies within the
    sums' rounding of a binary32 rounding boundary."""

    def __init__(self, steps: Mapping[int, Any], exchange: HaloExchange, sync: Callable[[], None] | None = None,
                 group: Any = None):
        self.steps = dict(steps)
        self.x = exchange
        self.sync = sync
        self.group = group
        first = next(iter(self.steps.values()))
        self.mass = bool(getattr(getattr(first, "cfg", None), "apmasscon", False)) and hasattr(first, "step_begin")
        if getattr(getattr(first, "cfg", None), "apmasscon", False) and not self.mass:
            from .errors import refuse  # noqa: PLC0415

            refuse(code="GM1B-DECOMPOSE-APMASSCON", gate="decomposition", option="apmasscon", value=True,
                   reason="the dry-air mass correction is a domain-wide reduction and this step runs as one call",
                   remedy="decompose with MoistLargeStep (its step splits at the ledger) or apmasscon=False")
        if self.mass:
            self._mass_setup()

    def _window(self, rank: int) -> tuple[int, int, int, int]:
        s = self.x.subs[rank]
        return (s.hw, s.hw + s.nx, s.hs, s.hs + s.ny)

    def _sum(self, parts: Mapping[int, Any]):
        import torch.distributed as dist  # noqa: PLC0415

        ranks = sorted(parts)
        total = parts[ranks[0]].clone()
        for r in ranks[1:]:
            total.add_(parts[r])
        if dist.is_available() and dist.is_initialized() and dist.get_world_size(self.group) > 1:
            dist.all_reduce(total, group=self.group)
        return total

    def _mass_setup(self) -> None:
        import torch  # noqa: PLC0415

        from .kessler import apmasscon_partials_words, dry_mass_from_partials, dry_mass_partials  # noqa: PLC0415

        first = next(iter(self.steps.values()))
        nk = first.cfg.nk
        self.cells = sum(s.nx * s.ny for s in self.x.subs.values()) * nk
        words = apmasscon_partials_words(nk)
        self.partials = {r: torch.zeros(words, dtype=torch.float64, device=st.s["rho"].device)
                         for r, st in self.steps.items()}
        for r, st in self.steps.items():
            s, m = st.s, st.m
            dry_mass_partials(s["rho"], s["ruh"], s["rvh"], m["rmh"], ni=st.cfg.ni, nj=st.cfg.nj, nk=nk,
                              window=self._window(r), partials=self.partials[r])
        total = self._sum(self.partials)
        for st in self.steps.values():
            dry_mass_from_partials(total, nk, st.s["mass1"])

    def step(self) -> None:
        if self.mass:
            for r, s in self.steps.items():
                s.step_begin(self._window(r), self.partials[r])
            total = self._sum(self.partials)
            for s in self.steps.values():
                s.step_end(total, self.cells)
        else:
            for s in self.steps.values():
                s.step()
        if self.sync is not None:
            self.sync()
        self.x.exchange()


def interior_slices(name: str, shape: tuple[int, ...], sub: Subdomain) -> tuple[slice, ...]:
    """Index slices of a subdomain's interior cells in its widened array."""
    xa, ya = _axes(name, shape, sub.eni, sub.enj)
    sl = [slice(None)] * len(shape)
    if xa is not None:
        off = _GHOSTS[shape[xa] - sub.eni]
        sl[xa] = slice(sub.hw + off, sub.hw + off + sub.nx)
    if ya is not None:
        off = _GHOSTS[shape[ya] - sub.enj]
        sl[ya] = slice(sub.hs + off, sub.hs + off + sub.ny)
    return tuple(sl)


def interior(arrays: Mapping[str, Any], sub: Subdomain, names: Iterable[str]) -> dict[str, np.ndarray]:
    """The interior cells of a subdomain's widened arrays (host copies)."""
    out = {}
    for n in names:
        a = arrays[n]
        a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
        out[n] = np.array(a[interior_slices(n, a.shape, sub)], order="C", copy=True)
    return out


def global_interior(arrays: Mapping[str, Any], ni: int, nj: int, sub: Subdomain, names: Iterable[str]):
    """The same cells of the single domain's arrays."""
    out = {}
    for n in names:
        a = arrays[n]
        a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
        xa, ya = _axes(n, a.shape, ni, nj)
        sl = [slice(None)] * a.ndim
        if xa is not None:
            off = _GHOSTS[a.shape[xa] - ni]
            sl[xa] = slice(sub.x0 + off, sub.x0 + off + sub.nx)
        if ya is not None:
            off = _GHOSTS[a.shape[ya] - nj]
            sl[ya] = slice(sub.y0 + off, sub.y0 + off + sub.ny)
        out[n] = np.ascontiguousarray(a[tuple(sl)])
    return out


def local_steps(cfg, host: Mapping[str, np.ndarray], metrics: Mapping[str, np.ndarray], subs: list[Subdomain],
                ranks: Iterable[int], make_step: Callable[[Any, dict, dict], Any]) -> dict[int, Any]:
    """{rank: step} for the subdomains of `ranks`: each built by
    make_step(subdomain config, widened state, widened metrics) from the
    global host state and metrics (the subdomain config is cfg with the
    widened ni, nj)."""
    import dataclasses  # noqa: PLC0415

    out = {}
    for s in subs:
        if s.rank not in ranks:
            continue
        sub_cfg = dataclasses.replace(cfg, ni=s.eni, nj=s.enj)
        out[s.rank] = make_step(sub_cfg, window(host, cfg.ni, cfg.nj, s), window(metrics, cfg.ni, cfg.nj, s))
    return out
