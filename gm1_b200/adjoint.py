"""Reverse-mode gradients on B200: the hand-written adjoint kernels of
libgm1b.so behind torch.autograd, and the differentiable warm-rain transport
model they serve.

The reference has no adjoint.  What is differentiated here is this library's
own forward operators, each with its adjoint kernel:

  advection_tendency   the open-filled carrier (pack + bcs, src/cm1core/
                       cuda_sound3_open_boundary.py:249-335, one launch) + the
                       whole-domain fifth-order / WENO5 tendency
                       (cpu_scalar_advection5_inplace, src/cm1core/cuda_advection5.py:
                       440), mass fluxes frozen; adjoint
                       gm1b_scalar_advection5_adjoint_open (face coefficients,
                       then a gather that folds the fill's transpose)
  kessler_collection   autoconversion + accretion with the qc limiter
                       (cpu_gm1_kessler_local_inplace, src/cm1core/cuda_gm1_kessler_local.py:
                       251); adjoint gm1b_kessler_collection_adjoint
  satadj1              the equation-set-1 saturation adjustment of the Kessler
                       driver (_cpu_satadj, src/cm1core/cuda_gm1_kessler_driver.py:
                       337-428); adjoint gm1b_satadj1_adjoint
  tridiagonal_solve    per-column Thomas solve (the acoustic column's implicit
                       w-pi' system, cuda_sound3_periodic.py:824-1027); its
                       adjoint is the transposed solve

WarmRainTransport composes them: per large step, theta', qv, qc and qr each
take the three RK stages s_n = s_0 + dt_n T_n(s_{n-1}) of the scalar RK
(nrk = 1, 2, 3; WENO5 at the third) under frozen mass fluxes, then qc and
qr are clipped at zero and collection and satadj1 act on the cell.  Gradients of any scalar objective
of the final state with respect to the initial state come back through the
adjoint kernels; ``checkpoint=True`` stores only the state at each large-step
boundary and recomputes the step's forward during the backward pass.

Subgradients at switches: the WENO-Z |b1 - b3| at b1 = b3 and the 1e30 cap
take 0, upstrpd's limiter and every Kessler limiter take the branch the
binary32 forward took, qr^0.875 is gated off at qr = 0.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any, Mapping

import torch
import torch.utils.checkpoint

from . import _native
from .advection import launch_cuda_scalar_advection5, padded_shapes
from .autotune import Autotuner
from .periodic import rk_stage_dt_f32

NG = 3
STATE_NAMES = ("th3d", "qv", "qc", "qr")
FLUX_NAMES = ("rru", "rrv", "rrw")
METRIC_NAMES = ("c1", "c2", "rr0", "gz", "divx")
THERMO_NAMES = ("th0", "pi0", "pp3d", "prs")


class _AdjArrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("scalar", "rru", "rrv", "rrw", "c1", "c2", "rr0", "gz", "divx",
                                               "tendency_adjoint", "scalar_adjoint")]


def _lib() -> ctypes.CDLL:
    lib = _native.lib()
    if not getattr(lib, "_adjoint_bound", False):
        i32, f32, vp, sz = ctypes.c_int32, ctypes.c_float, ctypes.c_void_p, ctypes.c_size_t
        lib.gm1b_scalar_advection5_adjoint.argtypes = [i32, i32, i32, ctypes.POINTER(_AdjArrays), i32, i32, f32, f32,
                                                       f32, ctypes.c_double, ctypes.c_uint32, vp, vp]
        lib.gm1b_scalar_advection5_adjoint_open.argtypes = [i32, i32, i32, ctypes.POINTER(_AdjArrays), i32, i32, f32,
                                                            f32, f32, ctypes.c_double, f32, vp, vp, vp, vp]
        lib.gm1b_scalar_advection5_adjoint_workspace_bytes.argtypes = [i32, i32, i32]
        lib.gm1b_scalar_advection5_adjoint_workspace_bytes.restype = sz
        lib.gm1b_scalar_carrier_open.argtypes = [i32, i32, i32, vp, vp, vp]
        ptr4 = ctypes.POINTER(vp)
        lib.gm1b_warm_rain_cell.argtypes = [sz, vp, vp, vp, vp, ptr4, ptr4, f32, vp]
        lib.gm1b_warm_rain_cell_adjoint.argtypes = [sz, vp, vp, vp, vp, ptr4, ptr4, ptr4, f32, vp]
        lib.gm1b_open_fill_scalar_adjoint.argtypes = [i32, i32, i32, vp, vp]
        lib.gm1b_tridiagonal_solve.argtypes = [i32, sz, vp, vp, vp, vp, vp, vp, i32, vp]
        lib.gm1b_kessler_collection.argtypes = [sz, vp, vp, f32, vp]
        lib.gm1b_kessler_collection_adjoint.argtypes = [sz, vp, vp, vp, vp, f32, vp]
        lib.gm1b_satadj1.argtypes = [sz] + [vp] * 7 + [vp]
        lib.gm1b_satadj1_adjoint.argtypes = [sz] + [vp] * 10 + [vp]
        for n in ("gm1b_scalar_advection5_adjoint", "gm1b_scalar_advection5_adjoint_open", "gm1b_scalar_carrier_open",
                  "gm1b_open_fill_scalar_adjoint", "gm1b_tridiagonal_solve",
                  "gm1b_kessler_collection", "gm1b_kessler_collection_adjoint", "gm1b_satadj1",
                  "gm1b_satadj1_adjoint", "gm1b_warm_rain_cell", "gm1b_warm_rain_cell_adjoint"):
            getattr(lib, n).restype = i32
        lib._adjoint_bound = True
    return lib


def _ptr(t: torch.Tensor, name: str) -> int:
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor")
    return t.data_ptr()


def _stream(device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


@dataclass(frozen=True)
class FrozenFlow:
    """The frozen transport and thermodynamic fields of one warm-rain run:
    mass fluxes rru (nk+2, nj+6, ni+7), rrv (nk+2, nj+7, ni+6), rrw (nk+3,
    nj+6, ni+6); c1, c2 (nk+1, nj, ni); rr0, divx, th0, pi0, pp3d, prs (nk,
    nj, ni); gz (nj, ni).  All sides open (CM1 wbc = ebc = sbc = nbc = 2)."""

    ni: int
    nj: int
    nk: int
    dx: float
    dy: float
    dz: float
    weps: float
    fields: Mapping[str, torch.Tensor]

    def __post_init__(self):
        sh = padded_shapes(self.ni, self.nj, self.nk)
        want = {"rru": sh["u"], "rrv": sh["v"], "rrw": sh["w"], "c1": sh["face"], "c2": sh["face"],
                "rr0": sh["cell"], "gz": (self.nj, self.ni), "divx": sh["cell"]}
        want.update({n: sh["cell"] for n in THERMO_NAMES})
        for n, shape in want.items():
            t = self.fields.get(n)
            if t is None:
                raise ValueError(f"missing frozen field {n}")
            _ptr(t, n)
            if tuple(t.shape) != shape:
                raise ValueError(f"{n} must have shape {shape}, got {tuple(t.shape)}")


LATERAL_OPEN = (2, 2, 2, 2)
OBC_OPEN = 0x2222


def _tendency(flow: FrozenFlow, padded: torch.Tensor, nrk: int, weps: float, chunk: int | None = None) -> torch.Tensor:
    f = flow.fields
    ten = torch.empty((flow.nk, flow.nj, flow.ni), dtype=torch.float32, device=padded.device)
    launch_cuda_scalar_advection5(
        padded, {n: f[n] for n in FLUX_NAMES}, {n: f[n] for n in ("c1", "c2", "rr0", "gz")}, f["divx"], ten, None,
        ni=flow.ni, nj=flow.nj, nk=flow.nk, nrk=nrk, dx=flow.dx, dy=flow.dy, dz=flow.dz, weps=weps,
        lateral_sides=LATERAL_OPEN, write_fluxes=False, levels_per_chunk=chunk)
    return ten


def _carrier(flow: FrozenFlow, scalar: torch.Tensor) -> torch.Tensor:
    """The compact scalar in its open-filled padded carrier (one launch)."""
    ni, nj, nk = flow.ni, flow.nj, flow.nk
    padded = torch.empty(padded_shapes(ni, nj, nk)["scalar"], dtype=torch.float32, device=scalar.device)
    _native.check(_lib().gm1b_scalar_carrier_open(ni, nj, nk, _ptr(scalar, "scalar"), padded.data_ptr(),
                                                  _stream(scalar.device)), "gm1b_scalar_carrier_open")
    return padded


def _adjoint_arrays(flow: FrozenFlow, scalar: torch.Tensor, lam: torch.Tensor, out: torch.Tensor) -> _AdjArrays:
    f = flow.fields
    return _AdjArrays(scalar=_ptr(scalar, "scalar"), rru=f["rru"].data_ptr(), rrv=f["rrv"].data_ptr(),
                      rrw=f["rrw"].data_ptr(), c1=f["c1"].data_ptr(), c2=f["c2"].data_ptr(), rr0=f["rr0"].data_ptr(),
                      gz=f["gz"].data_ptr(), divx=f["divx"].data_ptr(), tendency_adjoint=_ptr(lam, "tendency_adjoint"),
                      scalar_adjoint=out.data_ptr())


def _workspace(flow: FrozenFlow, device) -> torch.Tensor:
    n = _lib().gm1b_scalar_advection5_adjoint_workspace_bytes(flow.ni, flow.nj, flow.nk) // 4
    return torch.empty(n, dtype=torch.float32, device=device)


def advection_tendency_adjoint(flow: FrozenFlow, scalar: torch.Tensor, tendency_adjoint: torch.Tensor, nrk: int, *,
                               weps: float | None = None, scale: float = 1.0,
                               accumulate: torch.Tensor | None = None,
                               running_sum: torch.Tensor | None = None,
                               out: torch.Tensor | None = None) -> torch.Tensor:
    """dJ/d(compact scalar) for dJ/d(tendency) = scale * tendency_adjoint, the
    tendency taken on the compact scalar's open-filled carrier (the carrier
    is read through the fill's index map; a face-coefficient pass, then one
    gather per compact cell that folds the fill's transpose), plus
    ``accumulate`` when given; with ``running_sum`` the result comes back
    bare and running_sum receives accumulate + result (into ``out`` when
    given)."""
    ni, nj, nk = flow.ni, flow.nj, flow.nk
    lam = tendency_adjoint.contiguous()
    if out is None:
        out = torch.empty((nk, nj, ni), dtype=torch.float32, device=scalar.device)
    elif not out.is_contiguous() or tuple(out.shape) != (nk, nj, ni) or out.dtype != torch.float32:
        raise ValueError("out must be a contiguous float32 (nk, nj, ni) tensor")
    a = _adjoint_arrays(flow, scalar.contiguous(), lam, out)
    work = _workspace(flow, scalar.device)
    _native.check(_lib().gm1b_scalar_advection5_adjoint_open(
        ni, nj, nk, ctypes.byref(a), nrk, 1, flow.dx, flow.dy, flow.dz, flow.weps if weps is None else weps, scale,
        None if accumulate is None else _ptr(accumulate, "accumulate"),
        None if running_sum is None else _ptr(running_sum, "running_sum"), work.data_ptr(), _stream(scalar.device)),
        "gm1b_scalar_advection5_adjoint_open")
    return out


def advection_carrier_adjoint(flow: FrozenFlow, padded: torch.Tensor, tendency_adjoint: torch.Tensor, nrk: int, *,
                              weps: float | None = None) -> torch.Tensor:
    """dJ/d(carrier word), the whole padded (nk+2, nj+6, ni+6) array, for
    dJ/d(tendency) of the tendency on the padded scalar ``padded``."""
    lam = tendency_adjoint.contiguous()
    out = torch.empty_like(padded)
    a = _adjoint_arrays(flow, padded, lam, out)
    work = _workspace(flow, padded.device)
    _native.check(_lib().gm1b_scalar_advection5_adjoint(
        flow.ni, flow.nj, flow.nk, ctypes.byref(a), nrk, 1, flow.dx, flow.dy, flow.dz,
        flow.weps if weps is None else weps, OBC_OPEN, work.data_ptr(), _stream(padded.device)),
        "gm1b_scalar_advection5_adjoint")
    return out


class _AdvectionTendency(torch.autograd.Function):
    @staticmethod
    def forward(ctx, scalar, flow, nrk, weps, chunk):
        scalar = scalar.contiguous()
        ctx.save_for_backward(scalar)
        ctx.flow, ctx.nrk, ctx.weps = flow, nrk, weps
        return _tendency(flow, _carrier(flow, scalar), nrk, weps, chunk)

    @staticmethod
    def backward(ctx, grad):
        (scalar,) = ctx.saved_tensors
        return advection_tendency_adjoint(ctx.flow, scalar, grad, ctx.nrk, weps=ctx.weps), None, None, None, None


def advection_tendency(scalar: torch.Tensor, flow: FrozenFlow, nrk: int, weps: float | None = None,
                       levels_per_chunk: int | None = None) -> torch.Tensor:
    """The open-sided fifth-order (nrk 1, 2) / WENO5 (nrk 3) tendency of a
    compact (nk, nj, ni) scalar, differentiable in the scalar; ``weps`` the
    WENO epsilon (default: the flow's); ``levels_per_chunk`` the forward
    kernel's z-chunk (None: the library default)."""
    if nrk not in (1, 2, 3):
        raise ValueError("nrk must be one of 1, 2, 3")
    return _AdvectionTendency.apply(scalar, flow, nrk, float(flow.weps if weps is None else weps), levels_per_chunk)


class _Collection(torch.autograd.Function):
    @staticmethod
    def forward(ctx, qc, qr, dt):
        qc0, qr0 = qc.contiguous(), qr.contiguous()
        qc1, qr1 = qc0.clone(), qr0.clone()
        _native.check(_lib().gm1b_kessler_collection(qc1.numel(), _ptr(qc1, "qc"), _ptr(qr1, "qr"), dt,
                                                     _stream(qc1.device)), "gm1b_kessler_collection")
        ctx.save_for_backward(qc0, qr0)
        ctx.dt = dt
        return qc1, qr1

    @staticmethod
    def backward(ctx, gc, gr):
        qc0, qr0 = ctx.saved_tensors
        gc1, gr1 = gc.contiguous().clone(), gr.contiguous().clone()
        _native.check(_lib().gm1b_kessler_collection_adjoint(qc0.numel(), qc0.data_ptr(), qr0.data_ptr(),
                                                             gc1.data_ptr(), gr1.data_ptr(), ctx.dt,
                                                             _stream(qc0.device)), "gm1b_kessler_collection_adjoint")
        return gc1, gr1, None


def kessler_collection(qc: torch.Tensor, qr: torch.Tensor, dt: float) -> tuple[torch.Tensor, torch.Tensor]:
    """(qc', qr') after autoconversion and accretion over dt; differentiable."""
    if not dt > 0.0:
        raise ValueError("dt must be > 0")
    return _Collection.apply(qc, qr, float(dt))


class _Satadj1(torch.autograd.Function):
    @staticmethod
    def forward(ctx, th3d, qv, qc, th0, pi0, pp3d, prs):
        ins = [t.contiguous() for t in (th3d, qv, qc)]
        outs = [t.clone() for t in ins]
        frozen = [t.contiguous() for t in (th0, pi0, pp3d, prs)]
        ptrs = [_ptr(t, n) for t, n in zip(frozen, THERMO_NAMES)]
        _native.check(_lib().gm1b_satadj1(outs[0].numel(), *ptrs, *(t.data_ptr() for t in outs),
                                          _stream(th3d.device)), "gm1b_satadj1")
        ctx.save_for_backward(*ins, *frozen)
        return tuple(outs)

    @staticmethod
    def backward(ctx, g_th, g_qv, g_qc):
        th3d, qv, qc, th0, pi0, pp3d, prs = ctx.saved_tensors
        gs = [g.contiguous().clone() for g in (g_th, g_qv, g_qc)]
        _native.check(_lib().gm1b_satadj1_adjoint(th3d.numel(), th0.data_ptr(), pi0.data_ptr(), pp3d.data_ptr(),
                                                  prs.data_ptr(), th3d.data_ptr(), qv.data_ptr(), qc.data_ptr(),
                                                  *(g.data_ptr() for g in gs), _stream(th3d.device)),
                      "gm1b_satadj1_adjoint")
        return gs[0], gs[1], gs[2], None, None, None, None


def satadj1(th3d, qv, qc, th0, pi0, pp3d, prs) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """(th3d', qv', qc') after one equation-set-1 saturation adjustment at the
    frozen pressure; differentiable in th3d, qv, qc."""
    return _Satadj1.apply(th3d, qv, qc, th0, pi0, pp3d, prs)


class _Tridiagonal(torch.autograd.Function):
    @staticmethod
    def forward(ctx, a, b, c, d):
        a, b, c, d = (t.contiguous() for t in (a, b, c, d))
        x = torch.empty_like(d)
        work = torch.empty_like(d)
        n, cols = d.shape[0], d[0].numel()
        _native.check(_lib().gm1b_tridiagonal_solve(n, cols, _ptr(a, "a"), _ptr(b, "b"), _ptr(c, "c"), _ptr(d, "d"),
                                                    x.data_ptr(), work.data_ptr(), 0, _stream(d.device)),
                      "gm1b_tridiagonal_solve")
        ctx.save_for_backward(a, b, c, x)
        return x

    @staticmethod
    def backward(ctx, g):
        a, b, c, x = ctx.saved_tensors
        g = g.contiguous()
        y = torch.empty_like(g)
        work = torch.empty_like(g)
        n, cols = g.shape[0], g[0].numel()
        _native.check(_lib().gm1b_tridiagonal_solve(n, cols, a.data_ptr(), b.data_ptr(), c.data_ptr(), g.data_ptr(),
                                                    y.data_ptr(), work.data_ptr(), 1, _stream(g.device)),
                      "gm1b_tridiagonal_solve")
        # A x = d: dJ/dd = A^-T g; dJ/dA(k, m) = -y(k) x(m)
        ga = torch.zeros_like(a)
        gc = torch.zeros_like(c)
        ga[1:] = -y[1:] * x[:-1]
        gc[:-1] = -y[:-1] * x[1:]
        return ga, -y * x, gc, y


def tridiagonal_solve(a, b, c, d) -> torch.Tensor:
    """x with a(k) x(k-1) + b(k) x(k) + c(k) x(k+1) = d(k) per column; all four
    (n, ...) with level k first; differentiable in every coefficient."""
    if not (a.shape == b.shape == c.shape == d.shape) or d.dim() < 2 or d.shape[0] < 2:
        raise ValueError("a, b, c, d must share a shape (n >= 2, columns...)")
    return _Tridiagonal.apply(a, b, c, d)


class WarmRainTransport:
    """The differentiable warm-rain transport model on one device.

    ``step(state)`` maps the tuple (th3d, qv, qc, qr), each (nk, nj, ni)
    float32, to the next large step's; ``run(state, steps)`` repeats it,
    checkpointing each large step when ``checkpoint`` is set."""

    def __init__(self, flow: FrozenFlow, dt: float, *, weps: Mapping[str, float] | None = None,
                 checkpoint: bool = True, tuner: Autotuner | None = None):
        if not dt > 0.0:
            raise ValueError("dt must be > 0")
        self.flow = flow
        self.weps = tuple(float((weps or {}).get(n, flow.weps)) for n in STATE_NAMES)
        self.dt = float(dt)
        self.stage_dt = tuple(rk_stage_dt_f32(self.dt, nrk) for nrk in (1, 2, 3))
        self.checkpoint = checkpoint
        # the forward tendency's z-chunk per stage kind (fifth order at
        # nrk 1, 2; WENO5 at nrk 3), chosen for this grid by the tuner
        self.chunk = {1: None, 2: None, 3: None}
        if tuner is not None:
            sample = _carrier(flow, flow.fields["th0"])
            for nrk, kind in ((1, "scalar_advection5"), (3, "scalar_advection5_weno")):
                best = tuner.choose(kind, flow.ni, flow.nj, flow.nk,
                                    lambda c, nrk=nrk: _tendency(flow, sample, nrk, self.weps[0], c))
                self.chunk[nrk] = best
            self.chunk[2] = self.chunk[1]

    def step(self, th3d, qv, qc, qr):
        f = self.flow.fields
        new = []
        for s0, weps in zip((th3d, qv, qc, qr), self.weps):
            cur = s0
            for nrk in (1, 2, 3):
                cur = torch.add(s0, advection_tendency(cur, self.flow, nrk, weps, self.chunk[nrk]),
                                alpha=self.stage_dt[nrk - 1])
            new.append(cur)
        # the transport's undershoots clipped: the Kessler pieces take
        # non-negative water (the reference refuses qc, qr < 0)
        qc1, qr1 = kessler_collection(torch.clamp(new[2], min=0.0), torch.clamp(new[3], min=0.0), self.dt)
        th1, qv1, qc2 = satadj1(new[0], new[1], qc1, f["th0"], f["pi0"], f["pp3d"], f["prs"])
        return th1, qv1, qc2, qr1

    def run(self, state: tuple, steps: int) -> tuple:
        if steps < 1:
            raise ValueError("steps must be >= 1")
        cur = tuple(state)
        for _ in range(steps):
            if self.checkpoint and torch.is_grad_enabled():
                cur = torch.utils.checkpoint.checkpoint(self.step, *cur, use_reentrant=False)
            else:
                cur = self.step(*cur)
        return cur

    def vjp_step(self, state: tuple, adjoint: tuple) -> tuple:
        """One large step in reverse: the step recomputed from ``state`` (the
        checkpoint at its start), then ``adjoint`` (dJ/d of the step's
        output) pulled back to dJ/d of its input through the adjoint
        kernels.  A caller that keeps the step-boundary states of a forward
        sweep and runs this from the last step to the first gets the
        gradient of the whole window (what ``gradient`` does with
        torch.utils.checkpoint)."""
        leaves = tuple(t.detach().requires_grad_(True) for t in state)
        with torch.enable_grad():
            out = self.step(*leaves)
        return torch.autograd.grad(out, leaves, grad_outputs=tuple(adjoint))

    def gradient(self, state: Mapping[str, Any] | tuple, weights: Mapping[str, torch.Tensor] | tuple,
                 steps: int) -> tuple[torch.Tensor, tuple]:
        """J = sum over fields of <weights, final field>; returns (J, dJ/d state)."""
        if isinstance(state, Mapping):
            state = tuple(state[n] for n in STATE_NAMES)
        if isinstance(weights, Mapping):
            weights = tuple(weights[n] for n in STATE_NAMES)
        leaves = tuple(t.detach().clone().requires_grad_(True) for t in state)
        final = self.run(leaves, steps)
        j = sum((w * x).sum() for w, x in zip(weights, final))
        grads = torch.autograd.grad(j, leaves)
        return j.detach(), grads


class StageCheckpointedAdjoint:
    """The hand-written reverse of a WarmRainTransport step with checkpoints
    at the RK-stage boundaries.

    ``forward(x)`` runs the step and keeps each scalar's stage states
    s_1, s_2, s_3 (s_0 is the step's input): with those, the reverse needs
    no tendency recomputed: the advection adjoint reads each stage's
    open-filled carrier through the fill's index map.  ``reverse(saved, lam)``
    pulls dJ/d(step output) back to dJ/d(step input):

      satadj1 adjoint at (s_3 theta', s_3 qv, qc after collection),
      collection adjoint at the clipped s_3 qc, qr, the clip's mask
      (torch.clamp's: the gradient passes at 0), then per scalar
      lambda_0 = l_3 + l_2 + l_1 + T_1^T(s_0) dt_1 l_1 with
      l_2 = T_3^T(s_2) dt_3 l_3 and l_1 = T_2^T(s_1) dt_2 l_2,
      the dt scaling and the last sum fused into the gather kernel.

    The same gradient as the autograd path (up to the order of the float
    sums).  With ``streams`` > 1 the scalars' reverse chains (independent
    after the cell adjoint) run on that many side streams forked from the
    caller's stream and joined back (a CUDA graph capture keeps the fork);
    two at a time keep their face scratch in L2.  The words do not depend on
    it."""

    def __init__(self, model: WarmRainTransport, streams: int = 1):
        self.model = model
        dev = model.flow.fields["th0"].device
        self.streams = [torch.cuda.Stream(dev) for _ in range(streams)] if streams > 1 else []

    def forward(self, x: tuple) -> tuple[tuple, tuple]:
        m = self.model
        f = m.flow.fields
        stages = []
        new = []
        with torch.no_grad():
            for s0, weps in zip(x, m.weps):
                cur, kept = s0, [s0]
                for nrk in (1, 2, 3):
                    ten = _tendency(m.flow, _carrier(m.flow, cur), nrk, weps, m.chunk[nrk])
                    cur = torch.add(s0, ten, alpha=m.stage_dt[nrk - 1])
                    kept.append(cur)
                stages.append(tuple(kept))
                new.append(cur)
            out = tuple(torch.empty_like(t) for t in new)
            _warm_rain_cell(f, new, None, out, m.dt)
        return out, tuple(stages)

    def reverse(self, stages: tuple, lam: tuple) -> tuple:
        m = self.model
        f = m.flow.fields
        with torch.no_grad():
            l3s = tuple(torch.empty_like(st[3]) for st in stages)
            _warm_rain_cell(f, tuple(st[3] for st in stages), tuple(t.contiguous() for t in lam), l3s, m.dt)
            out = [torch.empty_like(l3) for l3 in l3s]
            main = torch.cuda.current_stream(l3s[0].device)
            for side in self.streams:
                side.wait_stream(main)
            for q, (st, l3, weps) in enumerate(zip(stages, l3s, m.weps)):
                with torch.cuda.stream(self.streams[q % len(self.streams)] if self.streams else main):
                    acc = torch.empty_like(l3)
                    # l2 = T_3^T dt_3 l3 with acc = l3 + l2; l1 = T_2^T dt_2 l2
                    # with acc += l1; lambda_0 = acc + T_1^T dt_1 l1
                    l2 = advection_tendency_adjoint(m.flow, st[2], l3, 3, weps=weps, scale=m.stage_dt[2],
                                                    accumulate=l3, running_sum=acc)
                    l1 = advection_tendency_adjoint(m.flow, st[1], l2, 2, weps=weps, scale=m.stage_dt[1],
                                                    accumulate=acc, running_sum=acc)
                    advection_tendency_adjoint(m.flow, st[0], l1, 1, weps=weps, scale=m.stage_dt[0], accumulate=acc,
                                               out=out[q])
            for side in self.streams:
                main.wait_stream(side)
        return tuple(out)


def _warm_rain_cell(f, state, lam, out, dt):
    """gm1b_warm_rain_cell (lam None) or its adjoint (lam = dJ/d(out), out
    receiving dJ/d(state))."""
    vp4 = ctypes.c_void_p * 4
    st = vp4(*(_ptr(t, "state") for t in state))
    o = vp4(*(_ptr(t, "out") for t in out))
    thermo = [_ptr(f[n], n) for n in THERMO_NAMES]
    stream = _stream(state[0].device)
    if lam is None:
        _native.check(_lib().gm1b_warm_rain_cell(state[0].numel(), *thermo, st, o, dt, stream), "gm1b_warm_rain_cell")
    else:
        lm = vp4(*(_ptr(t, "lam") for t in lam))
        _native.check(_lib().gm1b_warm_rain_cell_adjoint(state[0].numel(), *thermo, st, lm, o, dt, stream),
                      "gm1b_warm_rain_cell_adjoint")


class StepGraphs:
    """A model's plain forward step, its stage-saving forward step and the
    one-step reverse of StageCheckpointedAdjoint, each captured once as a
    CUDA graph over static flat buffers, so a sweep replays one graph per
    step instead of launching its kernels one by one, and moves each step's
    saved fields with one copy.

    Flat layouts, (n, nk, nj, ni) float32: the state (th3d, qv, qc, qr) is 4
    fields; a forward step's output is 16 (the next state, then s_1, s_2,
    s_3 of each scalar in state order); the reverse reads 20 (the step's
    input state, the 12 stage fields, dJ/d(step output)) and writes 4.
    ``gradient`` gives the words of the eager StageCheckpointedAdjoint."""

    def __init__(self, model: WarmRainTransport, like: tuple, streams: int = 2):
        self.model = model
        self.adjoint = StageCheckpointedAdjoint(model, streams=streams)
        dev = like[0].device
        shape = tuple(like[0].shape)
        self.xin = torch.stack([t.detach() for t in like]).contiguous()
        self.fout = torch.zeros((16,) + shape, dtype=torch.float32, device=dev)
        self.rin = torch.zeros((20,) + shape, dtype=torch.float32, device=dev)
        self.rin[:4].copy_(self.xin)
        self.rout = torch.zeros((4,) + shape, dtype=torch.float32, device=dev)
        self.sout = torch.zeros((4,) + shape, dtype=torch.float32, device=dev)
        x = tuple(self.xin[q] for q in range(4))
        stages_in = tuple((self.rin[q],) + tuple(self.rin[4 + 3 * q + r] for r in range(3)) for q in range(4))
        lam_in = tuple(self.rin[16 + q] for q in range(4))

        def fwd():
            y, stages = self.adjoint.forward(x)
            for q in range(4):
                self.fout[q].copy_(y[q])
                for r in range(3):
                    self.fout[4 + 3 * q + r].copy_(stages[q][r + 1])

        def rev():
            g = self.adjoint.reverse(stages_in, lam_in)
            for q in range(4):
                self.rout[q].copy_(g[q])

        def plain():
            with torch.no_grad():
                y = model.step(*x)
            for q in range(4):
                self.sout[q].copy_(y[q])

        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):  # first launches outside the capture
            for _ in range(2):
                plain()
                fwd()
                rev()
        torch.cuda.current_stream(dev).wait_stream(side)
        self.g_step, self.g_fwd, self.g_rev = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.g_step):
            plain()
        with torch.cuda.graph(self.g_fwd):
            fwd()
        with torch.cuda.graph(self.g_rev):
            rev()

    @staticmethod
    def stack(state: tuple) -> torch.Tensor:
        return torch.stack([t.detach() for t in state]).contiguous()

    def step(self, x: torch.Tensor) -> torch.Tensor:
        """The plain step of a stacked (4, nk, nj, ni) state."""
        self.xin.copy_(x)
        self.g_step.replay()
        return self.sout.clone()

    def forward(self, x: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """The stage-saving step of a stacked state: the (16, ...) block of
        the next state and the stage fields (into ``out`` when given: a
        sweep lays its whole checkpoint store out once)."""
        self.xin.copy_(x)
        self.g_fwd.replay()
        if out is None:
            return self.fout.clone()
        out.copy_(self.fout)
        return out

    def store(self, steps: int) -> torch.Tensor:
        """The checkpoint store of a ``steps``-step window: (steps, 16, nk,
        nj, ni) float32, 64 words per cell per step."""
        return torch.empty((steps,) + tuple(self.fout.shape), dtype=torch.float32, device=self.fout.device)

    def reverse(self, x: torch.Tensor, saved: torch.Tensor, lam: torch.Tensor) -> torch.Tensor:
        """dJ/d(stacked step input) from the step's input ``x``, its saved
        (16, ...) block and dJ/d(step output)."""
        self.rin[:4].copy_(x)
        self.rin[4:16].copy_(saved[4:])
        self.rin[16:].copy_(lam)
        self.g_rev.replay()
        return self.rout.clone()

    def gradient(self, state: tuple, weights: tuple, steps: int, store: torch.Tensor | None = None) -> tuple:
        """dJ/d state for J = sum <weights, final state>: a forward sweep
        keeping every step's stage block in ``store`` (made here when not
        given), then the reverse sweep."""
        store = self.store(steps) if store is None else store
        inputs, saved = [self.stack(state)], []
        for q in range(steps):
            saved.append(self.forward(inputs[-1], store[q]))
            inputs.append(saved[-1][:4])
        lam = self.stack(weights)
        for q in reversed(range(steps)):
            lam = self.reverse(inputs[q], saved[q], lam)
        return tuple(lam[q] for q in range(4))
