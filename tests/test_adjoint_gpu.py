"""The hand-written adjoint kernels on the GPU.

Forward pieces: collection and the single-pass saturation adjustment against
the reference's own outputs (golden fixtures), the tridiagonal solve against
a dense solve.  Adjoints: each kernel against binary64 autograd of the
restatements in oracle/adjoint_f64.py at the same point (bars stated per
test), the open-fill transpose word for word; then the whole differentiable
warm-rain transport: its gradient against binary64 autograd of the same
composition and against 16 central finite differences in binary64, and
checkpointed against stored activations word for word."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200 import adjoint as adj
from oracle import adjoint_f64 as f64
from tests._golden import load_npz
from tests.adjoint_common import NG, filled_carrier, warm_rain_case

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
WARM_RAIN_TAGS = ["warm_rain_8x6x5", "warm_rain_7x9x6"]


def _g(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(DEV)


def _t(a):
    return torch.from_numpy(np.asarray(a, np.float64).copy())


def _flow(fr, g):
    return adj.FrozenFlow(g["ni"], g["nj"], g["nk"], g["dx"], g["dy"], g["dz"], g["weps"],
                          {n: _g(v) for n, v in fr.items()})


def _ulps(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ia = a.astype(np.float32).view(np.int32).astype(np.int64)
    ib = b.astype(np.float32).view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
    ib = np.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
    return np.abs(ia - ib)


@pytest.mark.parametrize("tag", WARM_RAIN_TAGS)
def test_collection_forward_matches_reference(tag):
    """powf (CUDA) against numpy's binary32 power (the reference): every
    cell without rain is bit-exact; the others agree within 2 ulps of the
    input word (where the qc limiter is active the output qc is the rounding
    residual qc - (qc ar/t + qc cr/t), a few ulps of qc with either sign)."""
    meta, i, o = load_npz(tag)
    qc, qr = adj.kessler_collection(_g(i["coll_qc"]), _g(i["coll_qr"]), meta["dt"])
    for got, want, word in ((qc, o["coll_qc"], i["coll_qc"]), (qr, o["coll_qr"], o["coll_qr"])):
        got = got.cpu().numpy()
        assert np.count_nonzero(_ulps(got, want)[i["coll_qr"] == 0]) == 0
        diff = np.abs(got.astype(np.float64) - want)
        assert np.all(diff <= 2 * np.spacing(np.abs(word))), float(diff.max())


@pytest.mark.parametrize("tag", WARM_RAIN_TAGS)
def test_satadj1_forward_matches_reference(tag):
    """expf (CUDA) against numpy's binary32 exp (the reference): th3d, qv and
    qc within 1e-5 of the adjustment (one ulp of esl moves th3d by about
    1e-6 K through qvs - qv), three words in five identical at least."""
    _, i, o = load_npz(tag)
    th, qv, qc = adj.satadj1(*(_g(i[f"sat_{n}"]) for n in ("th3d", "qv", "qc", "th0", "pi0", "pp3d", "prs")))
    same = 0
    for name, got in (("th3d", th), ("qv", qv), ("qc", qc)):
        want = o[f"sat_{name}"]
        change = float(np.abs(want.astype(np.float64) - i[f"sat_{name}"]).max())
        err = float(np.abs(got.cpu().numpy().astype(np.float64) - want).max())
        assert err <= 1e-5 * change, (name, err, change)
        same += int(np.count_nonzero(got.cpu().numpy() == want))
    assert same >= 0.6 * 3 * i["sat_qv"].size


def test_tridiagonal_forward_and_transpose_match_dense_solves():
    rng = np.random.default_rng(2)
    n, cols = 12, 300
    a, c = rng.uniform(-1, 1, (n, cols)), rng.uniform(-1, 1, (n, cols))
    b = 3.0 + rng.random((n, cols))
    d = rng.standard_normal((n, cols))
    x = adj.tridiagonal_solve(*(_g(v) for v in (a, b, c, d))).cpu().numpy()
    lib = adj._lib()
    y = torch.empty((n, cols), dtype=torch.float32, device=DEV)
    work = torch.empty_like(y)
    ga, gb, gc, gd = (_g(v) for v in (a, b, c, d))
    assert lib.gm1b_tridiagonal_solve(n, cols, ga.data_ptr(), gb.data_ptr(), gc.data_ptr(), gd.data_ptr(),
                                      y.data_ptr(), work.data_ptr(), 1, None) == 0
    yt = y.cpu().numpy()
    for q in range(0, cols, 37):
        m = np.diag(b[:, q]) + np.diag(a[1:, q], -1) + np.diag(c[:-1, q], 1)
        assert np.abs(x[:, q] - np.linalg.solve(m, d[:, q])).max() <= 1e-5
        assert np.abs(yt[:, q] - np.linalg.solve(m.T, d[:, q])).max() <= 1e-5


def test_tridiagonal_gradient_matches_binary64_autograd():
    rng = np.random.default_rng(3)
    n, cols = 9, 40
    vals = [rng.uniform(-1, 1, (n, cols)), 3.0 + rng.random((n, cols)), rng.uniform(-1, 1, (n, cols)),
            rng.standard_normal((n, cols))]
    w = rng.standard_normal((n, cols))
    dev = [_g(v).requires_grad_(True) for v in vals]
    (adj.tridiagonal_solve(*dev) * _g(w)).sum().backward()
    ref = [_t(v).requires_grad_(True) for v in vals]
    (f64.tridiagonal_solve(*ref) * _t(w)).sum().backward()
    for name, p, q in zip("abcd", dev, ref):
        gp, gq = p.grad.cpu().numpy(), q.grad.numpy()
        if name == "a":
            gp, gq = gp[1:], gq[1:]
        if name == "c":
            gp, gq = gp[:-1], gq[:-1]
        assert np.abs(gp - gq).max() <= 1e-5 * np.abs(gq).max(), name


def test_open_fill_adjoint_is_the_transpose():
    ni, nj, nk = 11, 9, 8
    rng = np.random.default_rng(4)
    g = rng.standard_normal((nk + 2, nj + 2 * NG, ni + 2 * NG)).astype(np.float32)
    s = torch.zeros(g.shape, dtype=torch.float64, requires_grad=True)
    (f64.open_fill_scalar(s, ni, nj, nk) * _t(g)).sum().backward()
    want = s.grad.numpy()
    q = _g(g)
    assert adj._lib().gm1b_open_fill_scalar_adjoint(ni, nj, nk, q.data_ptr(), None) == 0
    got = q.cpu().numpy()
    # each edge word sums at most 1 + 3 + 3 + 9 halo words in binary32
    assert np.abs(got - want).max() <= 2e-6 * np.abs(want).max()


def test_carrier_fill_on_the_device_matches_the_host_fill():
    state, fr, g = warm_rain_case(ni=12, nj=10, nk=9, seed=5)
    flow = _flow(fr, g)
    got = adj._carrier(flow, _g(state["qc"])).cpu().numpy()
    assert np.array_equal(got, filled_carrier(state["qc"], 12, 10, 9))


@pytest.mark.parametrize("nrk", [1, 2, 3])
def test_advection_adjoint_matches_binary64_autograd(nrk):
    state, fr, g = warm_rain_case(ni=16, nj=12, nk=10, seed=7)
    ni, nj, nk = g["ni"], g["nj"], g["nk"]
    flow = _flow(fr, g)
    padded = filled_carrier(state["qv"], ni, nj, nk)
    lam = np.random.default_rng(8).standard_normal((nk, nj, ni)).astype(np.float32)
    # the kernel alone (before the fill transpose), on the filled carrier
    out = adj.advection_carrier_adjoint(flow, _g(padded), _g(lam), nrk).cpu().numpy()
    s = _t(padded).requires_grad_(True)
    ten = f64.scalar_advection5(s, *(_t(fr[n]) for n in ("rru", "rrv", "rrw", "c1", "c2", "rr0", "gz", "divx")),
                                nrk=nrk, dx=g["dx"], dy=g["dy"], dz=g["dz"], weps=g["weps"], obc=adj.OBC_OPEN)
    (ten * _t(lam)).sum().backward()
    want, got = s.grad.numpy(), out
    err = np.abs(got - want).max() / np.abs(want).max()
    print("nrk", nrk, "max relative error", err)
    # binary32 face adjoints (lam * rr0 * gz * rd) against binary64: 1e-5 of scale
    assert err <= 1e-5


def _relative(a: torch.Tensor, b: torch.Tensor) -> float:
    return float((a.double().cpu() - b.double().cpu()).norm() / b.double().cpu().norm())


@pytest.mark.parametrize("steps", [1, 3])
def test_warm_rain_gradient_matches_binary64_and_finite_differences(steps):
    state, fr, g = warm_rain_case(ni=16, nj=12, nk=10, seed=11)
    flow = _flow(fr, g)
    dt = 5.0
    model = adj.WarmRainTransport(flow, dt)
    rng = np.random.default_rng(12)
    weights = {n: rng.standard_normal(v.shape).astype(np.float32) for n, v in state.items()}
    j, grads = model.gradient({n: _g(v) for n, v in state.items()}, {n: _g(w) for n, w in weights.items()}, steps)
    frozen = {n: _t(v) for n, v in fr.items()}
    kw = dict(ni=g["ni"], nj=g["nj"], nk=g["nk"], dt=dt, dx=g["dx"], dy=g["dy"], dz=g["dz"], weps=g["weps"],
              steps=steps)

    def objective(x):
        out = f64.warm_rain_transport(x, frozen, **kw)
        return sum((_t(weights[n]) * out[n]).sum() for n in adj.STATE_NAMES)

    x0 = {n: _t(v).requires_grad_(True) for n, v in state.items()}
    j64 = objective(x0)
    g64 = torch.autograd.grad(j64, [x0[n] for n in adj.STATE_NAMES])
    # the binary32 trajectory: theta' rides on th0 near 300 K (an ulp of
    # 3e-5 K), so J is held to 1e-6 of sum |w x|, not of its cancelled sum
    with torch.no_grad():
        out64 = f64.warm_rain_transport({n: _t(v) for n, v in state.items()}, frozen, **kw)
        mass = float(sum((_t(weights[n]).abs() * out64[n].abs()).sum() for n in adj.STATE_NAMES))
    assert abs(float(j) - float(j64)) <= 1e-6 * mass
    errs = {n: _relative(gd, gr) for n, gd, gr in zip(adj.STATE_NAMES, grads, g64)}
    print("steps", steps, "relative L2 gradient error", errs)
    # binary32 trajectory and adjoint against binary64: 1e-4 per field (L2)
    assert max(errs.values()) <= 1e-4, errs
    # 16 central differences of the binary64 objective, each against the
    # binary32 adjoint's directional derivative, relative to |g| |v|.  The
    # step is 1e-8 of each field's scale: the saturation adjustment's
    # cloud-water limit and the clip at zero are kinks that wider steps
    # straddle (at 1e-6 a few cells do, and the difference quotient averages
    # the two sides), and binary64 leaves 1e-8 far above its rounding.
    scale = {n: float(np.abs(v).max()) + 1e-6 for n, v in state.items()}
    gnorm = float(sum(gr.double().cpu().norm() ** 2 * scale[n] ** 2 for n, gr in zip(adj.STATE_NAMES, grads)) ** 0.5)
    worst = 0.0
    for _ in range(16):
        v = {n: _t(rng.standard_normal(a.shape)) * scale[n] for n, a in state.items()}
        h = 1e-8
        with torch.no_grad():
            jp = objective({n: x0[n].detach() + h * v[n] for n in x0})
            jm = objective({n: x0[n].detach() - h * v[n] for n in x0})
        fd = float(jp - jm) / (2 * h)
        ad = sum(float((gr.double().cpu() * v[n]).sum()) for n, gr in zip(adj.STATE_NAMES, grads))
        worst = max(worst, abs(fd - ad) / gnorm)
    print("worst directional error / (|g| |v|)", worst)
    assert worst <= 1e-4


def test_checkpointed_gradient_is_word_identical_to_stored_activations():
    state, fr, g = warm_rain_case(ni=16, nj=12, nk=10, seed=13)
    flow = _flow(fr, g)
    rng = np.random.default_rng(14)
    weights = {n: _g(rng.standard_normal(v.shape)) for n, v in state.items()}
    x = {n: _g(v) for n, v in state.items()}
    _, g_ck = adj.WarmRainTransport(flow, 5.0, checkpoint=True).gradient(x, weights, 4)
    _, g_st = adj.WarmRainTransport(flow, 5.0, checkpoint=False).gradient(x, weights, 4)
    for a, b in zip(g_ck, g_st):
        assert torch.equal(a, b)


def test_refusals():
    state, fr, g = warm_rain_case(ni=12, nj=10, nk=9, seed=5)
    flow = _flow(fr, g)
    with pytest.raises(ValueError):
        adj.advection_tendency(_g(state["qv"]), flow, 4)
    with pytest.raises(ValueError):
        adj.WarmRainTransport(flow, 0.0)
    bad = dict(flow.fields)
    bad["rru"] = bad["rru"][:, :, :-1].contiguous()
    with pytest.raises(ValueError):
        adj.FrozenFlow(12, 10, 9, 1000.0, 1000.0, 400.0, 1e-6, bad)
    with pytest.raises(ValueError):
        adj.tridiagonal_solve(*(torch.zeros(1, 4, device=DEV) for _ in range(4)))


def test_stepwise_reverse_sweep_equals_the_checkpointed_gradient():
    """Forward sweep storing each large-step boundary, then vjp_step from the
    last step to the first: the same words as torch.utils.checkpoint."""
    state, fr, g = warm_rain_case(ni=16, nj=12, nk=10, seed=15)
    flow = _flow(fr, g)
    model = adj.WarmRainTransport(flow, 5.0, weps={"th3d": 1e-5, "qv": 1e-20, "qc": 1e-20, "qr": 1e-20})
    rng = np.random.default_rng(16)
    weights = tuple(_g(rng.standard_normal(state[n].shape)) for n in adj.STATE_NAMES)
    x = tuple(_g(state[n]) for n in adj.STATE_NAMES)
    ckpt = [x]
    with torch.no_grad():
        for _ in range(3):
            ckpt.append(model.step(*ckpt[-1]))
    lam = weights
    for q in reversed(range(3)):
        lam = model.vjp_step(ckpt[q], lam)
    _, ref = model.gradient(x, weights, 3)
    for a, b in zip(lam, ref):
        assert torch.equal(a, b)


def test_fused_carrier_gives_the_pack_and_fill_words():
    from gm1_b200.moist_ops import open_fill, pack_scalar  # noqa: PLC0415

    state, fr, g = warm_rain_case(ni=13, nj=11, nk=9, seed=17)
    flow = _flow(fr, g)
    s = _g(state["th3d"])
    want = torch.zeros((11, 17, 19), dtype=torch.float32, device=DEV)
    pack_scalar(s, want, ni=13, nj=11, nk=9)
    open_fill(want, "scalar", ni=13, nj=11, nk=9)
    assert torch.equal(adj._carrier(flow, s), want)


@pytest.mark.parametrize("nrk", [1, 3])
def test_compact_advection_adjoint_folds_the_fill(nrk):
    """dJ/d(compact scalar) through carrier fill and tendency, against
    binary64 autograd of pack, open fill and tendency."""
    state, fr, g = warm_rain_case(ni=16, nj=12, nk=10, seed=18)
    ni, nj, nk = g["ni"], g["nj"], g["nk"]
    flow = _flow(fr, g)
    lam = np.random.default_rng(19).standard_normal((nk, nj, ni)).astype(np.float32)
    # qv: no clipped zeros, so no stencil sits exactly on a limiter kink
    # (where the kernel's stated subgradient and torch's may differ)
    got = adj.advection_tendency_adjoint(flow, _g(state["qv"]), _g(lam), nrk).cpu().numpy()
    s = _t(state["qv"]).requires_grad_(True)
    p = f64.open_fill_scalar(f64.pack(s, ni, nj, nk), ni, nj, nk)
    ten = f64.scalar_advection5(p, *(_t(fr[n]) for n in ("rru", "rrv", "rrw", "c1", "c2", "rr0", "gz", "divx")),
                                nrk=nrk, dx=g["dx"], dy=g["dy"], dz=g["dz"], weps=g["weps"], obc=adj.OBC_OPEN)
    (ten * _t(lam)).sum().backward()
    want = s.grad.numpy()
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()


def test_tuned_model_gives_the_untuned_words():
    from gm1_b200.autotune import Autotuner  # noqa: PLC0415

    state, fr, g = warm_rain_case(ni=16, nj=12, nk=10, seed=20)
    flow = _flow(fr, g)
    x = tuple(_g(state[n]) for n in adj.STATE_NAMES)
    tuned = adj.WarmRainTransport(flow, 5.0, tuner=Autotuner())
    plain = adj.WarmRainTransport(flow, 5.0)
    with torch.no_grad():
        a, b = tuned.step(*x), plain.step(*x)
    for u, v in zip(a, b):
        assert torch.equal(u, v)


def test_stage_checkpointed_reverse_matches_autograd():
    """The hand-written reverse with RK-stage checkpoints against the
    autograd path through the same kernels: the same forward words, and the
    gradient within 1e-6 (relative L2; the two sum the stage adjoints in
    different orders)."""
    state, fr, g = warm_rain_case(ni=16, nj=12, nk=10, seed=21)
    flow = _flow(fr, g)
    model = adj.WarmRainTransport(flow, 5.0)
    rng = np.random.default_rng(22)
    weights = tuple(_g(rng.standard_normal(state[n].shape)) for n in adj.STATE_NAMES)
    x = tuple(_g(state[n]) for n in adj.STATE_NAMES)
    sc = adj.StageCheckpointedAdjoint(model)
    cur, saved = x, []
    for _ in range(3):
        cur, stages = sc.forward(cur)
        saved.append(stages)
    with torch.no_grad():
        ref = x
        for _ in range(3):
            ref = model.step(*ref)
    for a, b in zip(cur, ref):
        assert torch.equal(a, b)
    lam = weights
    for stages in reversed(saved):
        lam = sc.reverse(stages, lam)
    _, want = model.gradient(x, weights, 3)
    for a, b in zip(lam, want):
        assert _relative(a, b) <= 1e-6


def test_graph_replayed_sweep_gives_the_eager_words():
    state, fr, g = warm_rain_case(ni=16, nj=12, nk=10, seed=23)
    flow = _flow(fr, g)
    model = adj.WarmRainTransport(flow, 5.0)
    rng = np.random.default_rng(24)
    weights = tuple(_g(rng.standard_normal(state[n].shape)) for n in adj.STATE_NAMES)
    x = tuple(_g(state[n]) for n in adj.STATE_NAMES)
    graphs = adj.StepGraphs(model, x)
    got = graphs.gradient(x, weights, 3)
    sc = adj.StageCheckpointedAdjoint(model)
    cur, saved = x, []
    for _ in range(3):
        cur, stages = sc.forward(cur)
        saved.append(stages)
    want = weights
    for stages in reversed(saved):
        want = sc.reverse(stages, want)
    for a, b in zip(got, want):
        assert torch.equal(a, b)
    with torch.no_grad():
        plain = model.step(*x)
    stepped = graphs.step(adj.StepGraphs.stack(x))
    for q, b in enumerate(plain):
        assert torch.equal(stepped[q], b)
    del graphs
