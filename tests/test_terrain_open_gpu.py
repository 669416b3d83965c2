"""Parity of the CUDA terrain/open acoustic stage through the C ABI with the
reference's CPU twin (golden fixtures: every array after every RK stage, the
eight ablations, alph/kdiv) and with the oracle on multi-tile and minimum
grids, with and without the diagnostic scratch words.  Bar: every float32
word identical."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gm1_b200 import terrain_open as tos
from gm1_b200._native import Gm1bError
from oracle import terrain_open as orc
from tests.golden.make_golden import terrain_open_fixture
from tests.test_oracle_terrain_open import PARAMS, TAGS, digest, load

pytestmark = pytest.mark.gpu

PROGNOSTIC = tuple(n for n in tos.COMPARE_OUTPUT_NAMES if n not in tos.COLUMN_DIAGNOSTIC_NAMES) + ("scalar",)


def _dev(d):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in d.items()}


def _digests(dev):
    torch.cuda.synchronize()
    return {n: digest(dev[n].cpu().numpy()) for n in tos.ALL_ARRAY_NAMES}


def _bad(got: dict, want: dict, names) -> list[str]:
    out = []
    for n in names:
        g = got[n].cpu().numpy() if isinstance(got[n], torch.Tensor) else got[n]
        w = want[n]
        if not np.array_equal(g.view(np.uint32), w.view(np.uint32)):
            k = int(np.count_nonzero(g.view(np.uint32) != w.view(np.uint32)))
            out.append(f"{n}({k})")
    return out


@pytest.mark.parametrize("tag", TAGS)
def test_stages_bit_exact_vs_reference(tag):
    meta, a, m, want = load(tag)
    p = {k: meta[k] for k in PARAMS}
    dev, mdev = _dev(a), _dev(m)
    for stage in meta["stages"]:
        r = tos.launch_cuda_psolver3_terrain_open_stage(dev, mdev, nrk=stage["nrk"], **p)
        assert r.cadence[0]["nloop"] == stage["nloop"]
        got = _digests(dev)
        assert sorted(n for n in got if got[n] != stage["digests"][n]) == [], f"nrk={stage['nrk']}"
    assert _bad(dev, want, tos.ALL_ARRAY_NAMES) == []


@pytest.mark.parametrize("name", list(orc.ABLATION_BITS))
def test_each_ablation_bit_exact_vs_reference(name):
    meta, a, m, _ = load("tos_reftest_5x4x5")
    p = {k: meta[k] for k in PARAMS}
    dev, mdev = _dev(a), _dev(m)
    tos.launch_cuda_psolver3_terrain_open_three_stage(
        dev, mdev, ablations=tos.TerrainOpenSoundAblations(**{name: False}), **p)
    got = _digests(dev)
    assert sorted(n for n in got if got[n] != meta["ablations"][name][n]) == []


def test_alph_kdiv_bit_exact_vs_reference():
    meta, a, m, _ = load("tos_seeded_9x7x8")
    p = {k: meta[k] for k in PARAMS}
    ak = meta["alph_kdiv"]
    dev, mdev = _dev(a), _dev(m)
    for stage in ak["stages"]:
        tos.launch_cuda_psolver3_terrain_open_stage(dev, mdev, nrk=stage["nrk"], alph=ak["alph"], kdiv=ak["kdiv"], **p)
        got = _digests(dev)
        assert sorted(n for n in got if got[n] != stage["digests"][n]) == []


@pytest.mark.parametrize("ni,nj,nk,nsound,dz", [(70, 37, 20, 6, 250.0), (45, 66, 12, 8, 333.3), (3, 3, 4, 6, 200.0),
                                               (33, 5, 41, 4, 480.0)])
def test_three_stages_bit_exact_vs_oracle(ni, nj, nk, nsound, dz):
    a, m = terrain_open_fixture(ni, nj, nk, 7 + ni + nj)
    p = dict(ni=ni, nj=nj, nk=nk, dt=2.0, nsound=nsound, dx=450.0, dy=520.0, dz=dz)
    ref = {k: v.copy() for k, v in a.items()}
    orc.terrain_open_three_stage(ref, m, **p)
    dev, mdev = _dev(a), _dev(m)
    tos.launch_cuda_psolver3_terrain_open_three_stage(dev, mdev, **p)
    torch.cuda.synchronize()
    assert _bad(dev, ref, tos.ALL_ARRAY_NAMES) == []


def test_compact_mode_prognostics_match_and_skip_scratch():
    ni, nj, nk = 70, 37, 20
    a, m = terrain_open_fixture(ni, nj, nk, 11)
    p = dict(ni=ni, nj=nj, nk=nk, dt=2.0, nsound=6, dx=450.0, dy=520.0, dz=250.0)
    ref = {k: v.copy() for k, v in a.items()}
    orc.terrain_open_three_stage(ref, m, **p)
    compact = {k: v for k, v in a.items()}
    for n in tos.COLUMN_DIAGNOSTIC_NAMES:
        compact[n] = np.full((1,), 7.0, np.float32)
    dev, mdev = _dev(compact), _dev(m)
    tos.launch_cuda_psolver3_terrain_open_three_stage(
        dev, mdev, compiled=tos.compile_cuda_psolver3_terrain_open(retain_column_diagnostics=False), **p)
    torch.cuda.synchronize()
    assert _bad(dev, ref, PROGNOSTIC) == []
    assert all(float(dev[n][0]) == 7.0 for n in tos.COLUMN_DIAGNOSTIC_NAMES)


def test_oversized_column_refused_by_the_library():
    ni, nj, nk = 4, 4, 161
    a, m = terrain_open_fixture(ni, nj, nk, 3)
    dev, mdev = _dev(a), _dev(m)
    with pytest.raises(Gm1bError, match="nk"):
        tos.launch_cuda_psolver3_terrain_open_three_stage(dev, mdev, ni=ni, nj=nj, nk=nk, dt=2.0, nsound=6, dx=1.0,
                                                          dy=1.0, dz=100.0)


def _column(lv, m, ni, nj, nk):
    from gm1_b200.momentum import StretchedMomentumColumn
    from tests.test_oracle_momentum import _padded_rho0

    rho0p = _padded_rho0(m["rho0_3d"], ni, nj, nk)
    t = lambda x: torch.from_numpy(np.array(x, dtype=np.float32)).cuda()  # noqa: E731
    vertical = StretchedMomentumColumn(False, None, sigma=t(lv.sigma), sigmaf=t(lv.sigmaf), rds=t(lv.rds),
                                       rdsf=t(lv.rdsf), ztop=lv.ztop_m)
    host = {"sigma": lv.sigma, "sigmaf": lv.sigmaf, "rds": lv.rds, "rdsf": lv.rdsf, "ztop": lv.ztop_m,
            "rho0p": rho0p}
    return vertical, host, t(rho0p)


@pytest.mark.parametrize("ni,nj,nk,spec", [(37, 21, 10, (1100.0, 40.0, 700.0)), (70, 9, 14, (1630.0, 40.0, 1030.0)),
                                           (3, 3, 10, (1100.0, 40.0, 700.0))])
def test_stretched_terrain_stage_matches_oracle(ni, nj, nk, spec):
    """launch_cuda_gm1_child_psolver3_open_stage on a generated stretched
    column (20 m at the ground to 200 m aloft) and a horizontally varying
    padded base density: every array, scratch included, word-identical to the
    oracle restatement after each of the three RK stages."""
    from gm1_b200.vertical import build_vertical_levels

    lv = build_vertical_levels(stretch_z=1, nk=nk, dz_m=100.0, ztop_m=spec[0], str_bot_m=spec[1],
                               str_top_m=spec[2], dz_bot_m=20.0, dz_top_m=200.0)
    a, m = terrain_open_fixture(ni, nj, nk, 300 + ni)
    vertical, host, rho0p = _column(lv, m, ni, nj, nk)
    p = dict(ni=ni, nj=nj, nk=nk, dt=2.0, nsound=6, dx=450.0, dy=520.0)
    ref = {k: v.copy() for k, v in a.items()}
    dev, mdev = _dev(a), _dev(m)
    mdev["rho0_padded"] = rho0p
    for nrk in (1, 2, 3):
        orc.terrain_open_stage_column(ref, m, host, nrk=nrk, **p)
        r = tos.launch_cuda_gm1_child_psolver3_open_stage(dev, mdev, nrk=nrk, vertical=vertical, **p)
        r.ready_event.synchronize()
        assert _bad(dev, ref, tos.ALL_ARRAY_NAMES) == [], f"nrk={nrk}"


def test_stretched_terrain_stage_on_a_uniform_column_is_the_uniform_stage():
    from gm1_b200.vertical import uniform_vertical_levels

    ni, nj, nk, dz = 40, 11, 12, 250.0
    a, m = terrain_open_fixture(ni, nj, nk, 5)
    m["rho0_3d"][:] = m["rho0_3d"][:, :1, :1]
    vertical, _, rho0p = _column(uniform_vertical_levels(nk, dz), m, ni, nj, nk)
    p = dict(ni=ni, nj=nj, nk=nk, dt=2.0, nsound=6, dx=450.0, dy=520.0)
    one, two, mdev = _dev(a), _dev(a), _dev(m)
    mdev["rho0_padded"] = rho0p
    tos.launch_cuda_psolver3_terrain_open_three_stage(one, mdev, dz=dz, **p)
    for nrk in (1, 2, 3):
        tos.launch_cuda_gm1_child_psolver3_open_stage(two, mdev, nrk=nrk, vertical=vertical, **p)
    torch.cuda.synchronize()
    assert _bad(two, {k: v.cpu().numpy() for k, v in one.items()}, tos.ALL_ARRAY_NAMES) == []


def test_stretched_terrain_stage_refusals():
    from gm1_b200.momentum import StretchedMomentumColumn
    from gm1_b200.vertical import uniform_vertical_levels

    ni, nj, nk = 9, 8, 6
    a, m = terrain_open_fixture(ni, nj, nk, 5)
    vertical, _, rho0p = _column(uniform_vertical_levels(nk, 200.0), m, ni, nj, nk)
    dev, mdev = _dev(a), _dev(m)
    p = dict(ni=ni, nj=nj, nk=nk, nrk=1, dt=2.0, nsound=6, dx=450.0, dy=520.0)
    with pytest.raises(ValueError, match="rho0_padded"):
        tos.launch_cuda_gm1_child_psolver3_open_stage(dev, mdev, vertical=vertical, **p)
    mdev["rho0_padded"] = rho0p
    with pytest.raises(ValueError, match="vertical mh"):
        tos.launch_cuda_gm1_child_psolver3_open_stage(dev, mdev, vertical=StretchedMomentumColumn(True, None), **p)
    with pytest.raises(ValueError, match="sigmaf"):
        bad = StretchedMomentumColumn(False, None, sigma=vertical.sigma, sigmaf=vertical.sigmaf, rds=vertical.rds,
                                      rdsf=vertical.rdsf, ztop=vertical.ztop + 10.0)
        tos.launch_cuda_gm1_child_psolver3_open_stage(dev, mdev, vertical=bad, **p)
    with pytest.raises(ValueError, match="four sides"):
        tos.launch_cuda_gm1_child_psolver3_open_stage(dev, mdev, vertical=vertical, lateral_sides=(1, 1, 2, 2), **p)


@pytest.mark.parametrize("ni,nj,nk,sides", [(37, 21, 10, (2, 2, 2, 2)), (70, 9, 14, (1, 1, 2, 2)),
                                            (33, 40, 10, (2, 2, 1, 1)), (3, 3, 10, (1, 1, 1, 1))])
def test_flat_stretched_stage_matches_oracle(ni, nj, nk, sides):
    """The flat column's stage (sound.F's terrain_flag=.false. texts) on
    rdz*mh / rdz*mf of a generated stretched column, on four lateral
    families: every array, scratch included, word-identical to the oracle
    restatement after each of the three RK stages."""
    from gm1_b200.momentum import StretchedMomentumColumn, momentum_open_boundary_code
    from tests.test_oracle_terrain_open import _flat_column

    col = _flat_column(nk)
    a, m = terrain_open_fixture(ni, nj, nk, 500 + ni)
    t = lambda x: torch.from_numpy(np.array(x, dtype=np.float32)).cuda()  # noqa: E731
    vertical = StretchedMomentumColumn(True, None, mh=t(col["mh"]), mf=t(col["mf"]), rdz=col["rdz"])
    from tests.test_oracle_momentum import _padded_rho0

    p = dict(ni=ni, nj=nj, nk=nk, dt=2.0, nsound=6, dx=450.0, dy=520.0)
    ref = {k: v.copy() for k, v in a.items()}
    dev, mdev = _dev(a), _dev(m)
    mdev["rho0_padded"] = t(_padded_rho0(m["rho0_3d"], ni, nj, nk))
    for nrk in (1, 2, 3):
        orc.terrain_open_stage_flat(ref, m, col, nrk=nrk, obc=momentum_open_boundary_code(sides), **p)
        r = tos.launch_cuda_gm1_child_psolver3_open_stage(dev, mdev, nrk=nrk, vertical=vertical, lateral_sides=sides,
                                                          **p)
        r.ready_event.synchronize()
        assert _bad(dev, ref, tos.ALL_ARRAY_NAMES) == [], f"nrk={nrk}"


def test_flat_stretched_stage_replays_from_a_cuda_graph():
    """The stretched-column stage allocates nothing and synchronises nothing
    on a flat column: captured once in a CUDA graph and replayed, it leaves
    the same words as the eager launch."""
    from gm1_b200.momentum import StretchedMomentumColumn
    from tests.test_oracle_momentum import _padded_rho0
    from tests.test_oracle_terrain_open import _flat_column

    ni, nj, nk, sides = 40, 12, 10, (1, 1, 2, 2)
    col = _flat_column(nk)
    a, m = terrain_open_fixture(ni, nj, nk, 77)
    t = lambda x: torch.from_numpy(np.array(x, dtype=np.float32)).cuda()  # noqa: E731
    vertical = StretchedMomentumColumn(True, None, mh=t(col["mh"]), mf=t(col["mf"]), rdz=col["rdz"])
    p = dict(ni=ni, nj=nj, nk=nk, nrk=2, dt=2.0, nsound=6, dx=450.0, dy=520.0, vertical=vertical,
             lateral_sides=sides)
    eager, graphed, mdev = _dev(a), _dev(a), _dev(m)
    mdev["rho0_padded"] = t(_padded_rho0(m["rho0_3d"], ni, nj, nk))
    tos.launch_cuda_gm1_child_psolver3_open_stage(eager, mdev, **p)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # first call outside the capture configures the kernels
        warm = _dev(a)
        tos.launch_cuda_gm1_child_psolver3_open_stage(warm, mdev, **p)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        tos.launch_cuda_gm1_child_psolver3_open_stage(graphed, mdev, stream=torch.cuda.current_stream(), **p)
    g.replay()
    torch.cuda.synchronize()
    assert _bad(graphed, {k: v.cpu().numpy() for k, v in eager.items()}, tos.ALL_ARRAY_NAMES) == []
