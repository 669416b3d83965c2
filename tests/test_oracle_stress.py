"""The flat-column SGS stress oracle (oracle/stress_oracle.c) against the
reference's own CPU twin of the stress, cpu_sgs_stress_tendency_inplace
(src/cm1core/cuda_sgs_stress_tendency.py:292; goldens stress_*.npz written
by tests/golden/make_golden.py), and its size-independent properties.

The reference has no NumPy twin of the flat (terrain_flag=.false.) texts
the stretched column runs.  Their gettau forms t11/t22/t33/t13/t23 with the
twin's very statements, so those words are pinned bit for bit.  The flat
t12 sums its eight kmh pairwise and reads the nearest interior corner at an
open edge, and turbu/turbv/turbw group the same products differently (and
drop the terrain terms that are exact zeros on flat metrics).  So on the
level-uniform golden, where both texts form the same sums, the flat
tendencies match the twin's within rounding: max |err| <= 2e-5 of the
largest tendency added.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from oracle import stress as ost

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ("stress_7x6x5", "stress_9x8x7")


def _load(tag):
    z = np.load(GOLDEN / f"{tag}.npz")
    meta = json.loads(str(z["meta"]))
    inp = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    out = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return meta, inp, out


def _flat_arrays(meta, inp):
    ni, nj, nk = meta["ni"], meta["nj"], meta["nk"]
    a = {n: np.ascontiguousarray(inp[n]).copy() for n in ("s11", "s22", "s33", "s12", "s13", "s23", "kmh", "kmv",
                                                          "rho", "rf", "mh", "mf", "u3d", "v3d", "w3d", "uten",
                                                          "vten", "wten")}
    a.update(ost.zeros(ni, nj, nk, ost.TAU_NAMES))
    return a


@pytest.mark.parametrize("tag", CASES)
def test_gettau_words_the_flat_and_terrain_texts_share(tag):
    meta, inp, out = _load(tag)
    a = _flat_arrays(meta, inp)
    ost.flat_gettau(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"])
    for n in ("t11", "t22", "t33", "t13", "t23"):
        assert np.array_equal(a[n].view(np.uint32), out[n].view(np.uint32)), n
    # t12 on interior corners: the same eight coefficients summed in another order
    ni, nj = meta["ni"], meta["nj"]
    got, want = a["t12"][:, 1:nj, 1:ni], out["t12"][:, 1:nj, 1:ni]
    assert np.max(np.abs(got - want)) <= 4 * np.finfo(np.float32).eps * np.max(np.abs(want))


def test_momentum_stress_matches_the_twin_where_the_texts_form_the_same_sums():
    meta, inp, out = _load("stress_9x8x7")
    assert meta["level_uniform"]
    ni, nj, nk = meta["ni"], meta["nj"], meta["nk"]
    a = _flat_arrays(meta, inp)
    ost.flat_gettau(a, ni=ni, nj=nj, nk=nk)
    rdz = float(np.float32(1.0) / np.float32(meta["dz"]))
    ost.flat_momentum_stress(a, ni=ni, nj=nj, nk=nk, dx=meta["dx"], dy=meta["dy"], rdz=rdz, dt=meta["dt"])
    for n in ("uten", "vten", "wten"):
        added_flat = a[n].astype(np.float64) - inp[n]
        added_twin = out[n].astype(np.float64) - inp[n]
        if n == "wten":
            added_flat, added_twin = added_flat[1:nk], added_twin[1:nk]
        scale = np.max(np.abs(added_twin))
        assert scale > 0.0, n
        assert np.max(np.abs(added_flat - added_twin)) <= 2e-5 * scale, n
    # the twin leaves wten's boundary faces alone; so does the restatement
    assert np.array_equal(a["wten"][[0, nk]], inp["wten"][[0, nk]])


def _random_column(ni, nj, nk, seed):
    rng = np.random.default_rng(seed)
    sh = ost.stress_shapes(ni, nj, nk)
    f = np.float32
    a = {n: np.zeros(sh[n], f) for n in sh}
    a["rho"][:] = rng.uniform(0.5, 1.2, sh["rho"])
    a["rf"][:] = rng.uniform(0.5, 1.2, sh["rf"])
    mh = rng.uniform(0.6, 1.6, nk).astype(f)
    a["mh"][:] = mh[:, None, None]
    a["mh_profile"][1:nk + 1] = mh
    a["mf"][:] = rng.uniform(0.6, 1.6, nk + 1).astype(f)[:, None, None]
    a["kmh"][:] = rng.uniform(1.0, 30.0, sh["kmh"])
    a["kmv"][:] = rng.uniform(1.0, 30.0, sh["kmv"])
    return a


def test_a_uniform_wind_has_no_stress():
    """Zero strain and stress; the implicit solve returns the uniform wind
    to within its rounding, so the tendency is a few ulps of u / dt."""
    ni, nj, nk = 9, 7, 8
    a = _random_column(ni, nj, nk, 3)
    a["u3d"][:] = 7.5
    a["v3d"][:] = -3.25
    a["w3d"][:] = 0.0
    before = {n: a[n].copy() for n in ost.TENDENCY_NAMES}
    ost.flat_sgs_stress(a, ni=ni, nj=nj, nk=nk, dx=100.0, dy=100.0, rdz=0.01, dt=0.6)
    for n in ost.STRAIN_NAMES + ost.TAU_NAMES:
        assert not np.any(a[n]), n
    bound = 8 * np.spacing(np.float32(7.5)) / 0.6 * 2.0
    for n in ost.TENDENCY_NAMES:
        assert np.max(np.abs(a[n] - before[n])) <= bound, n


def test_zero_coefficients_leave_the_tendencies():
    ni, nj, nk = 8, 9, 7
    a = _random_column(ni, nj, nk, 4)
    rng = np.random.default_rng(5)
    for n in ("u3d", "v3d", "w3d"):
        a[n][:] = rng.normal(0.0, 2.0, a[n].shape)
    a["kmh"][:] = 0.0
    a["kmv"][:] = 0.0
    for n in ost.TENDENCY_NAMES:
        a[n][:] = rng.normal(0.0, 1e-3, a[n].shape)
    before = {n: a[n].copy() for n in ost.TENDENCY_NAMES}
    ost.flat_sgs_stress(a, ni=ni, nj=nj, nk=nk, dx=100.0, dy=100.0, rdz=0.01, dt=0.6)
    for n in ost.TENDENCY_NAMES:
        assert np.array_equal(a[n], before[n]), n


def test_a_sheared_u_alone_drives_only_u():
    """u = U(z) with horizontally uniform coefficients: t12, t22, t23 and
    t33 vanish and t13 is uniform on each level, so v and w get no
    tendency at all while u does."""
    ni, nj, nk = 6, 7, 10
    a = _random_column(ni, nj, nk, 6)
    a["kmh"][:] = a["kmh"][:, :1, :1]
    a["kmv"][:] = a["kmv"][:, :1, :1]
    a["rho"][:] = a["rho"][:, :1, :1]
    a["rf"][:] = a["rf"][:, :1, :1]
    a["u3d"][:] = np.linspace(0.0, 20.0, nk).astype(np.float32)[:, None, None] ** 1.5
    ost.flat_sgs_stress(a, ni=ni, nj=nj, nk=nk, dx=100.0, dy=100.0, rdz=0.01, dt=0.6)
    assert np.any(a["uten"])
    assert not np.any(a["vten"])
    assert not np.any(a["wten"])


# ------------------------------------------------------------------ turbs
# The reference's CPU twin of turbs, cpu_gm1_scalar_turbulence_inplace
# (src/cm1core/cuda_gm1_scalar_turbulence.py:414), runs the terrain texts;
# on flat metrics (gz = rgz = 1, zero slopes) with dx = dy = 128 m every
# product with 1/dx is exact and its terrain terms add exact zeros, so the
# flat text's words are the twin's: pinned bit for bit.
TURBS_CASES = ("turbs_8x7x6", "turbs_11x9x10")


@pytest.mark.parametrize("tag", TURBS_CASES)
def test_flat_turbs_is_the_twin_word_for_word(tag):
    meta, inp, out = _load(tag)
    a = {k: np.ascontiguousarray(v).copy() for k, v in inp.items()}
    ost.flat_scalar_turbulence(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], numq=6, dx=meta["dx"], dy=meta["dy"],
                               dz=meta["dz"], dt=meta["dt"])
    for n in ("thten1", "qten"):
        assert np.array_equal(a[n].view(np.uint32), out[n].view(np.uint32)), n
        assert np.any(a[n] != inp[n]), n


def test_turbs_of_uniform_scalars_only_rounds():
    """Horizontally and vertically uniform theta and moisture: no flux, and
    the implicit solve returns the field to within its rounding."""
    ni, nj, nk = 7, 6, 9
    rng = np.random.default_rng(9)
    f = np.float32
    a = {"th0": np.full(nk, 300.0, f), "tha": np.full((nk, nj, ni), 2.5, f),
         "qa": np.full((3, nk, nj, ni), 4.0e-3, f), "rho": rng.uniform(0.5, 1.1, (nk, nj, ni)).astype(f),
         "rf": rng.uniform(0.5, 1.1, (nk + 1, nj, ni)).astype(f), "mh": np.ones((nk, nj, ni), f),
         "mf": np.ones((nk + 1, nj, ni), f), "khh": rng.uniform(1, 50, (nk + 1, nj, ni)).astype(f),
         "khv": rng.uniform(1, 50, (nk + 1, nj, ni)).astype(f), "thten1": np.zeros((nk, nj, ni), f),
         "qten": np.zeros((3, nk, nj, ni), f)}
    a["rr"] = (f(1.0) / a["rho"]).astype(f)
    ost.flat_scalar_turbulence(a, ni=ni, nj=nj, nk=nk, numq=3, dx=100.0, dy=100.0, dz=50.0, dt=0.6)
    assert np.max(np.abs(a["thten1"])) <= 8 * np.spacing(f(2.5)) / 0.6 * 3.0
    assert np.max(np.abs(a["qten"])) <= 8 * np.spacing(f(4.0e-3)) / 0.6 * 3.0


# --------------------------------------------------------------- Rayleigh
# cpu_build_rayleigh_coefficients and cpu_rayleigh_held_inplace
# (src/cm1core/cuda_rayleigh_held.py:264, :213) on the reference's sealed
# damping selection: the coefficient builders (the oracle's and the
# package's host set-up) and the held tendencies pinned bit for bit.
RAYLEIGH_CASES = ("rayleigh_9x7x75", "rayleigh_6x8x75")


@pytest.mark.parametrize("tag", RAYLEIGH_CASES)
def test_rayleigh_coefficients_and_held_tendencies_are_the_twins(tag):
    from gm1_b200.rayleigh import build_rayleigh_coefficients

    z = np.load(GOLDEN / f"{tag}.npz")
    meta, inp, out = _load(tag)
    for tau in (ost.rayleigh_coefficients(z["zh"], z["zf"], damping_start_m=meta["damping_start_m"]),
                build_rayleigh_coefficients(z["zh"], z["zf"], damping_start_m=meta["damping_start_m"])):
        for got, name in zip(tau, ("tauh", "taus", "tauf")):
            assert np.array_equal(got.view(np.uint32), inp[name][:, 0, 0].view(np.uint32)), name
    assert np.count_nonzero(inp["tauh"][:, 0, 0]) > 0
    a = {k: np.ascontiguousarray(v).copy() for k, v in inp.items()}
    ost.rayleigh_held(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], rdalpha=meta["rdalpha"])
    for n in ("uten1", "vten1", "wten1", "thten1"):
        assert np.array_equal(a[n].view(np.uint32), out[n].view(np.uint32)), n
    # the column-profile layout gives the same words on laterally uniform tau
    b = {k: np.ascontiguousarray(v).copy() for k, v in inp.items()}
    for name in ("tauh", "taus", "tauf"):
        b[name] = np.ascontiguousarray(inp[name][:, 0, 0])
    ost.rayleigh_held(b, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], rdalpha=meta["rdalpha"], profiles=True)
    for n in ("uten1", "vten1", "wten1", "thten1"):
        assert np.array_equal(b[n].view(np.uint32), out[n].view(np.uint32)), n


def test_rayleigh_add_momentum_is_the_held_sum():
    meta, inp, out = _load("rayleigh_9x7x75")
    a = {k: np.ascontiguousarray(v).copy() for k, v in inp.items()}
    rng = np.random.default_rng(3)
    held = {n: rng.normal(0.0, 1e-3, a[n].shape).astype(np.float32) for n in ("uten1", "vten1", "wten1")}
    for n, v in held.items():
        a[n][:] = v
    ost.rayleigh_held(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], rdalpha=meta["rdalpha"], add_momentum=True)
    for n, v in held.items():
        assert np.array_equal(a[n], (out[n] + v).astype(np.float32)), n
    assert np.array_equal(a["thten1"], out["thten1"])


# ------------------------------------------------------ dissipative heating
def test_dissipative_heating_is_the_twins_cell_formula():
    """cpu_idiss_cell_f32 (src/cm1core/eqtset2_energy_terms.py:176), the
    reference's scalar mirror, cell by cell (golden idiss_7x6x9.npz)."""
    meta, inp, out = _load("idiss_7x6x9")
    a = {k: np.ascontiguousarray(v).copy() for k, v in inp.items()}
    ost.dissipative_heating(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"])
    assert np.array_equal(a["thten1"].view(np.uint32), out["thten1"].view(np.uint32))
    assert np.any(a["thten1"] != inp["thten1"])


# ------------------------------------------- the reference's own flat texts
# tests/golden/make_kernel_text_golden.py flat-stress runs the reference's
# CUDA texts of the flat stretched-column closure on the host (the strain
# passes, gettau, turbu/turbv/turbw and turbs with its pad/pack copies, the
# binary32 intrinsics as IEEE operations): the restatement is word-identical.
FLAT_TEXT_CASES = ("flat_stress_12x10x10", "flat_stress_9x13x14")


@pytest.mark.parametrize("tag", FLAT_TEXT_CASES)
def test_flat_stress_and_turbs_are_the_reference_texts_word_for_word(tag):
    z = np.load(GOLDEN / f"{tag}.npz")
    ni, nj, nk = (int(x) for x in z["meta"])
    dx, dy, dt, dz = (float(z[k]) for k in ("dx", "dy", "dt", "dz"))
    a = {k[3:]: np.ascontiguousarray(z[k]).copy() for k in z.files if k.startswith("in_")}
    rdz = float(a["rdz"].item())
    a.update(ost.zeros(ni, nj, nk, ost.STRAIN_NAMES + ost.TAU_NAMES))
    ost.flat_sgs_stress(a, ni=ni, nj=nj, nk=nk, dx=dx, dy=dy, rdz=rdz, dt=dt)
    for n in ost.STRAIN_NAMES + ost.TAU_NAMES + ost.TENDENCY_NAMES:
        got, want = a[n], z["out_" + n]
        if n in ("s13", "s23"):  # the texts write face levels 1..nk-1 only
            got, want = got[1:nk], want[1:nk]
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), n
    b = {k: a[k] for k in ost.SCALAR_TURBULENCE_INPUTS}
    b["thten1"], b["qten"] = a["thten1"].copy(), a["qten"].copy()
    ost.flat_scalar_turbulence(b, ni=ni, nj=nj, nk=nk, numq=3, dx=dx, dy=dy, dz=dz, dt=dt)
    for n in ("thten1", "qten"):
        assert np.array_equal(b[n].view(np.uint32), z["out_" + n].view(np.uint32)), n


# ------------------------------------------------------ the terrain texts
# The uniform column runs the terrain texts (gettau, turbu/turbv/turbw,
# turbs) the twins state: the restatements give their words bit for bit.
@pytest.mark.parametrize("tag", CASES)
def test_terrain_stress_is_the_twin_word_for_word(tag):
    meta, inp, out = _load(tag)
    ni, nj, nk = meta["ni"], meta["nj"], meta["nk"]
    a = {k: np.ascontiguousarray(v).copy() for k, v in inp.items()}
    ost.terrain_gettau(a, ni=ni, nj=nj, nk=nk)
    ost.terrain_momentum_stress(a, ni=ni, nj=nj, nk=nk, dx=meta["dx"], dy=meta["dy"], dz=meta["dz"], dt=meta["dt"])
    for n in ost.TAU_NAMES + ost.TENDENCY_NAMES:
        assert np.array_equal(a[n].view(np.uint32), out[n].view(np.uint32)), n
    for n in ost.TENDENCY_NAMES:
        assert np.any(a[n] != inp[n]), n


@pytest.mark.parametrize("tag", TURBS_CASES)
def test_terrain_turbs_is_the_twin_word_for_word(tag):
    meta, inp, out = _load(tag)
    a = {k: np.ascontiguousarray(v).copy() for k, v in inp.items()}
    ost.terrain_scalar_turbulence(a, ni=meta["ni"], nj=meta["nj"], nk=meta["nk"], numq=6, dx=meta["dx"],
                                  dy=meta["dy"], dz=meta["dz"], dt=meta["dt"])
    for n in ("thten1", "qten"):
        assert np.array_equal(a[n].view(np.uint32), out[n].view(np.uint32)), n
