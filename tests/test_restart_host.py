"""The CM1FCP1 restart envelope on the host: round trip of every dtype the
moist step carries, the refusals the reference's envelope reader makes (bad
magic, a header over the cap, a payload of the wrong length, bytes that miss
their SHA-256, a contract that misses its digest, another profile), and the
carried inventory: the oracle's composition written after 3 large steps,
read back into a fresh start and stepped 3 more is word-identical to 6
uninterrupted steps (the restart pair's contract, src/cm1core/
cartesian_restart.py:1-60)."""

from __future__ import annotations

import json
import struct
from types import SimpleNamespace

import numpy as np
import pytest

from gm1_b200.restart import CARRIED, HEADER_LIMIT_BYTES, MAGIC, RestartRefusal, read_envelope, write_envelope
from oracle.moist_composition import OracleMoistStep
from oracle.moist_initial import weisman_klemp_initial_state


def _arrays():
    rng = np.random.default_rng(1)
    return {"u": rng.standard_normal((3, 4, 5)).astype(np.float32), "budget": rng.standard_normal(10),
            "mask": (rng.random((2, 3)) > 0.5).astype(np.uint8), "neg_zero": np.array([-0.0, np.nan], np.float32)}


def test_round_trip_is_word_identical(tmp_path):
    a = _arrays()
    p = tmp_path / "r.cm1fcp"
    h = write_envelope(p, {"step": 7, "model_time_s": 4.2}, a)
    assert p.read_bytes()[:8] == MAGIC and h["payload_nbytes"] == sum(x.nbytes for x in a.values())
    header, back = read_envelope(p)
    assert header["step"] == 7 and header["model_time_s"] == 4.2
    assert list(back) == list(a)
    for n in a:
        assert back[n].dtype == a[n].dtype and back[n].shape == a[n].shape
        assert np.array_equal(back[n].view(np.uint8), a[n].view(np.uint8)), n


def _corrupt(p, offset, value):
    b = bytearray(p.read_bytes())
    b[offset] = value
    p.write_bytes(bytes(b))


def test_refusals(tmp_path):
    a = _arrays()
    p = tmp_path / "r.cm1fcp"
    write_envelope(p, {"step": 1}, a)
    good = p.read_bytes()
    length = struct.unpack("<Q", good[8:16])[0]
    # the magic
    _corrupt(p, 0, ord("X"))
    with pytest.raises(RestartRefusal, match="magic"):
        read_envelope(p)
    # a header over the cap
    p.write_bytes(good[:8] + struct.pack("<Q", HEADER_LIMIT_BYTES + 1) + good[16:])
    with pytest.raises(RestartRefusal, match="header"):
        read_envelope(p)
    # a payload of the wrong length
    p.write_bytes(good[:-3])
    with pytest.raises(RestartRefusal, match="payload"):
        read_envelope(p)
    # one payload byte flipped: its array misses its digest
    p.write_bytes(good)
    _corrupt(p, 16 + length + 5, good[16 + length + 5] ^ 0x40)
    with pytest.raises(RestartRefusal, match="SHA-256"):
        read_envelope(p)
    # a contract that no longer matches its digest
    header = json.loads(good[16:16 + length])
    header["contract"]["array_specs"][0]["shape"] = [3, 4, 6]
    raw = json.dumps(header, sort_keys=True).encode()
    p.write_bytes(good[:8] + struct.pack("<Q", len(raw)) + raw + good[16 + length:])
    with pytest.raises(RestartRefusal, match="digest"):
        read_envelope(p)
    # unsupported dtypes are refused on the way in
    with pytest.raises(RestartRefusal, match="dtype"):
        write_envelope(tmp_path / "c.cm1fcp", {}, {"c": np.zeros(2, np.complex64)})


@pytest.mark.parametrize("stretched", [False, True], ids=["uniform", "stretched"])
def test_carried_inventory_resumes_the_composition(tmp_path, stretched):
    column = SimpleNamespace(ztop_m=20800.0, str_bot_m=200.0, str_top_m=15800.0, dz_bot_m=20.0,
                             dz_top_m=500.0) if stretched else None
    ni, nj, nk, dx, dz, dt, ns = (12, 10, 80, 100.0, 100.0, 0.6, 8) if stretched else (14, 12, 12, 1000.0, 250.0, 5.0, 10)
    cfg = SimpleNamespace(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, dt=dt, nsound=ns, alph=0.60, kdiv=0.10,
                          lateral_sides=(2, 2, 2, 2), obc=0x2222, column=column)
    host, metrics = weisman_klemp_initial_state(cfg, seed=3, bubble_radius_m=(4 * dx, 4 * dz), bubble_center_z_m=4 * dz,
                                                bubble_cloud=1.0e-3, bubble_rain=5.0e-4)
    start = {k: v.copy() for k, v in host.items()}
    run = OracleMoistStep(cfg, host, {k: v.copy() for k, v in metrics.items()})
    for _ in range(3):
        run.step()
    p = tmp_path / "restart.cm1fcp"
    write_envelope(p, {"step": 3}, {n: run.s[n] for n in CARRIED})
    for _ in range(3):
        run.step()
    _, back = read_envelope(p)
    again = OracleMoistStep(cfg, start, {k: v.copy() for k, v in metrics.items()})
    for n in CARRIED:
        again.s[n][...] = back[n]
    for _ in range(3):
        again.step()
    for n, a in run.s.items():
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(again.s[n]).view(np.uint8)), n
