"""Helpers to read the golden fixtures made by tests/golden/make_golden.py."""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_npz(tag: str) -> tuple[dict, dict[str, np.ndarray], dict[str, np.ndarray]]:
    with np.load(GOLDEN / f"{tag}.npz") as z:
        meta = json.loads(str(z["meta"]))
        inputs = {k[3:]: z[k].copy() for k in z.files if k.startswith("in_")}
        outputs = {k[4:]: z[k].copy() for k in z.files if k.startswith("out_")}
    return meta, inputs, outputs


def load_json(name: str):
    return json.loads((GOLDEN / name).read_text())


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes(order="C")).hexdigest()


def bit_mismatches(expected: dict[str, np.ndarray], actual: dict[str, np.ndarray], names) -> dict[str, int]:
    bad = {}
    for name in names:
        e = expected[name].view(np.uint32)
        a = np.ascontiguousarray(actual[name]).view(np.uint32)
        if e.shape != a.shape:
            bad[name] = -1
            continue
        n = int(np.count_nonzero(e != a))
        if n:
            bad[name] = n
    return bad
