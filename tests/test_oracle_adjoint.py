"""Pins the binary64 restatements that the adjoint kernels are checked
against (oracle/adjoint_f64.py): the open fill against the reference's own
bcs output, collection and the single-pass saturation adjustment against the
reference's cpu_gm1_kessler_local_inplace and _cpu_satadj outputs, the
advection tendency against the word-pinned binary32 advection oracle, and
the tridiagonal solve against a dense solve.  Then the composed warm-rain
model's autograd gradient against central finite differences, both in
binary64."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import adjoint_f64 as f64
from oracle import advection as adv
from tests._golden import GOLDEN, load_npz
from tests.adjoint_common import filled_carrier, warm_rain_case

WARM_RAIN_TAGS = ["warm_rain_8x6x5", "warm_rain_7x9x6"]


def _t(a):
    return torch.from_numpy(np.asarray(a, np.float64).copy())


def test_open_fill_restatement_matches_reference_bcs():
    z = np.load(GOLDEN / "open_fills_9x7x6.npz")
    ni, nj, nk = 9, 7, 6
    got = f64.open_fill_scalar(_t(z["in_scalar"]), ni, nj, nk).numpy()
    assert np.array_equal(got.astype(np.float32), z["out_scalar"])


def test_host_carrier_fill_matches_restatement():
    rng = np.random.default_rng(1)
    s = rng.standard_normal((6, 7, 9)).astype(np.float32)
    want = f64.open_fill_scalar(f64.pack(_t(s), 9, 7, 6), 9, 7, 6).numpy().astype(np.float32)
    assert np.array_equal(filled_carrier(s, 9, 7, 6), want)


@pytest.mark.parametrize("tag", WARM_RAIN_TAGS)
def test_collection_restatement_matches_reference(tag):
    meta, i, o = load_npz(tag)
    qc, qr = f64.kessler_collection(_t(i["coll_qc"]), _t(i["coll_qr"]), meta["dt"])
    for got, want in ((qc, o["coll_qc"]), (qr, o["coll_qr"])):
        err = np.abs(got.numpy() - want.astype(np.float64))
        assert err.max() <= 2e-6 * max(float(np.abs(want).max()), 1e-12)


@pytest.mark.parametrize("tag", WARM_RAIN_TAGS)
def test_satadj1_restatement_matches_reference(tag):
    _, i, o = load_npz(tag)
    th, qv, qc = f64.satadj1(*(_t(i[f"sat_{n}"]) for n in ("th0", "pi0", "pp3d", "prs", "th3d", "qv", "qc")))
    # bar: 5e-5 of the largest adjustment.  The binary32 temperature (th0 +
    # th3d near 300 K, an ulp of 3e-5 K) moves qvs by about 1e-7 of itself,
    # and qvs - qv cancels to a tenth of qvs, so the reference's own words sit
    # about 2e-5 of the adjustment away from the binary64 value.
    for name, got in (("th3d", th), ("qv", qv), ("qc", qc)):
        want = o[f"sat_{name}"].astype(np.float64)
        change = float(np.abs(want - i[f"sat_{name}"]).max())
        err = float(np.abs(got.numpy() - want).max())
        assert err <= 5e-5 * change, (name, err, change)


@pytest.mark.parametrize("nrk", [1, 2, 3])
def test_advection_restatement_matches_binary32_oracle(nrk):
    state, fr, g = warm_rain_case(ni=12, nj=10, nk=9, seed=4)
    ni, nj, nk = g["ni"], g["nj"], g["nk"]
    padded = filled_carrier(state["qv"], ni, nj, nk)
    a = {"scalar": padded, "rru": fr["rru"], "rrv": fr["rrv"], "rrw": fr["rrw"], "c1": fr["c1"], "c2": fr["c2"],
         "rr0": fr["rr0"], "gz": fr["gz"], "divx": fr["divx"],
         "tendency": np.zeros((nk, nj, ni), np.float32), "flux_x": np.zeros_like(fr["rru"]),
         "flux_y": np.zeros_like(fr["rrv"]), "flux_z": np.zeros_like(fr["rrw"])}
    adv.scalar_advection5(a, ni=ni, nj=nj, nk=nk, nrk=nrk, dx=g["dx"], dy=g["dy"], dz=g["dz"], weps=g["weps"],
                          lateral_obc=0x2222)
    got = f64.scalar_advection5(_t(padded), *(_t(fr[n]) for n in ("rru", "rrv", "rrw", "c1", "c2", "rr0", "gz",
                                                                   "divx")),
                                nrk=nrk, dx=g["dx"], dy=g["dy"], dz=g["dz"], weps=g["weps"], obc=0x2222).numpy()
    want = a["tendency"].astype(np.float64)
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()


def test_tridiagonal_restatement_matches_dense_solve():
    rng = np.random.default_rng(2)
    n, cols = 7, 5
    a, c = rng.uniform(-1, 1, (n, cols)), rng.uniform(-1, 1, (n, cols))
    b = 3.0 + rng.random((n, cols))
    d = rng.standard_normal((n, cols))
    x = f64.tridiagonal_solve(*(torch.from_numpy(v) for v in (a, b, c, d))).numpy()
    for q in range(cols):
        m = np.diag(b[:, q]) + np.diag(a[1:, q], -1) + np.diag(c[:-1, q], 1)
        assert np.allclose(m @ x[:, q], d[:, q], rtol=0, atol=1e-12)


def test_warm_rain_restatement_gradient_matches_central_differences():
    state, fr, g = warm_rain_case(ni=10, nj=9, nk=8, seed=6)
    frozen = {n: _t(v) for n, v in fr.items()}
    kw = dict(ni=g["ni"], nj=g["nj"], nk=g["nk"], dt=5.0, dx=g["dx"], dy=g["dy"], dz=g["dz"], weps=g["weps"],
              steps=2)
    rng = np.random.default_rng(9)
    weights = {n: _t(rng.standard_normal(v.shape)) for n, v in state.items()}
    x0 = {n: _t(v).requires_grad_(True) for n, v in state.items()}

    def objective(x):
        out = f64.warm_rain_transport(x, frozen, **kw)
        return sum((weights[n] * out[n]).sum() for n in out)

    j = objective(x0)
    grads = torch.autograd.grad(j, list(x0.values()))
    scale = {n: float(np.abs(v).max()) + 1e-6 for n, v in state.items()}
    for q in range(4):
        v = {n: _t(rng.standard_normal(a.shape)) * scale[n] for n, a in state.items()}
        h = 1e-8  # narrower than the kinks' spacing (cloud-water limit, clip at zero)
        with torch.no_grad():
            jp = objective({n: x0[n] + h * v[n] for n in x0})
            jm = objective({n: x0[n] - h * v[n] for n in x0})
        fd = float(jp - jm) / (2 * h)
        ad = sum(float((gr * v[n]).sum()) for gr, n in zip(grads, x0))
        assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1.0), (q, fd, ad)
