"""Restart of the composed moist step: write a CM1FCP1 envelope, continue
from it word for word.

Behaviour followed (reference file:line):
  the restart pair's design - every array the model carries from one large
  step to the next is written, and read straight back into the same arrays
  with nothing recomputed; the base state is rebuilt from the same sounding
  and geometry and pinned by digest
      src/cm1core/cartesian_restart.py:1-60 (restart_write.F:364-839,
      README.namelist:1512-1516)
  the CM1FCP1 envelope - eight magic bytes b"CM1FCP1\\0", the header length
  as a little-endian u64, a JSON header (each array's offset, byte count and
  SHA-256, the contract's array specs and its digest, the payload length),
  then the payload of little-endian words; a header over 1 MiB, a payload of
  the wrong length or an array whose bytes miss their digest is refused
      src/cm1core/cartesian_restart.py:1048-1110, :197-210, :618-626
      src/cm1core/render_restart.py:46, :291-350

What this step carries (the inventory CM1's restart_write.F names, in this
build's array names): the step-start prognostics ua, va, wa, ppi, tha, qa,
tkea and ppx with their RK-stage twins u3d, v3d, w3d, pp3d, th3d, q3d; rho,
prs and the face density rf; the eqtset 2 rate carriers qpten, qtten, qvten,
qcten; the TKE dissipation dissten the next closure reads; the rain
accumulators rain and prate; the radiative lateral histories radbcw, radbce,
radbcs, radbcn; the FP64 budgets asq and qbudget; the dry-air mass ledger
mass1 of the final-RK mass correction (restart_write.F:412); and the scalars
step count and model time.  Everything else of the state is either rebuilt from the
configuration (the base state, whose SHA-256 the header records and a resume
checks) or scratch the next step overwrites before reading.
"""

from __future__ import annotations

import hashlib
import json
import os
import struct
from pathlib import Path
from typing import Any, Mapping

import numpy as np

from .errors import CM1Refusal

MAGIC = b"CM1FCP1\0"
HEADER_LIMIT_BYTES = 1024 * 1024
PROFILE = "gm1b.moist-restart/v1"

CARRIED = ("ua", "va", "wa", "ppi", "tha", "qa", "tkea", "ppx", "u3d", "v3d", "w3d", "pp3d", "th3d", "q3d", "rho",
           "prs", "rf", "qpten", "qtten", "qvten", "qcten", "dissten", "rain", "prate", "radbcw", "radbce", "radbcs",
           "radbcn", "asq", "qbudget", "mass1")
# the rebuilt base state a resume must find unchanged
BASE_STATE = ("th0", "pi0", "qv0", "th0_3d", "pi0_3d", "uh", "vh", "ruh", "rvh")
CONFIG_KEYS = ("ni", "nj", "nk", "dx", "dy", "dz", "dt", "nsound", "alph", "kdiv", "lateral_sides")
_DTYPES = {"float32": "<f4", "float64": "<f8", "uint8": "|u1", "int32": "<i4", "uint32": "<u4"}


class RestartRefusal(CM1Refusal):
    """A restart that cannot be written or continued from, with the reason."""


def _refuse(code: str, reason: str, remedy: str) -> None:
    raise RestartRefusal(code=code, gate="restart", option="restart", value=None, reason=reason, remedy=remedy)


def _digest(arrays: Mapping[str, np.ndarray], names) -> str:
    h = hashlib.sha256()
    for n in names:
        a = np.ascontiguousarray(arrays[n])
        h.update(n.encode() + b"\0" + str(a.dtype).encode() + b"\0" + repr(a.shape).encode() + b"\0")
        h.update(a.tobytes())
    return h.hexdigest()


def config_record(cfg) -> dict[str, Any]:
    """The configuration words a resume must match."""
    rec = {k: getattr(cfg, k) for k in CONFIG_KEYS}
    rec["lateral_sides"] = list(rec["lateral_sides"])
    col = getattr(cfg, "column", None)
    rec["column"] = None if col is None else {k: getattr(col, k) for k in
                                              ("ztop_m", "str_bot_m", "str_top_m", "dz_bot_m", "dz_top_m")}
    return rec


def write_envelope(path: str | os.PathLike, fields: Mapping[str, Any], arrays: Mapping[str, np.ndarray]) -> dict:
    """Write a CM1FCP1 envelope of host arrays (in the given order) with the
    header fields; written to a temporary name and renamed into place.
    Returns the header."""
    specs, rows, blobs, offset = [], [], [], 0
    for name, a in arrays.items():
        a = np.ascontiguousarray(a)
        if str(a.dtype) not in _DTYPES:
            _refuse("RESTART-DTYPE", f"{name} has dtype {a.dtype}, which the envelope does not carry",
                    "pass float32, float64, uint8, int32 or uint32 arrays")
        data = a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes()
        specs.append({"name": name, "shape": list(a.shape), "dtype": str(a.dtype)})
        rows.append({"name": name, "offset": offset, "nbytes": len(data), "sha256": hashlib.sha256(data).hexdigest()})
        blobs.append(data)
        offset += len(data)
    contract = {"profile": PROFILE, "array_specs": specs}
    header = dict(fields)
    header.update(contract=contract, contract_sha256=hashlib.sha256(
        json.dumps(contract, sort_keys=True).encode()).hexdigest(), arrays=rows, payload_nbytes=offset)
    raw = json.dumps(header, sort_keys=True).encode("utf-8")
    if len(raw) > HEADER_LIMIT_BYTES:
        _refuse("RESTART-HEADER", f"the header takes {len(raw)} bytes; the envelope caps it at {HEADER_LIMIT_BYTES}",
                "write fewer arrays")
    path = Path(path)
    tmp = path.with_name(path.name + ".partial")
    with open(tmp, "wb") as f:
        f.write(MAGIC + struct.pack("<Q", len(raw)))
        f.write(raw)
        for b in blobs:
            f.write(b)
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, path)
    return header


def read_envelope(path: str | os.PathLike) -> tuple[dict, dict[str, np.ndarray]]:
    """(header, arrays) of a CM1FCP1 envelope; every array's bytes checked
    against the SHA-256 its header records."""
    path = Path(path)
    size = path.stat().st_size
    with open(path, "rb") as f:
        prefix = f.read(16)
        if len(prefix) != 16 or prefix[:8] != MAGIC:
            _refuse("RESTART-ENVELOPE", f"{path} does not begin with the CM1FCP1 magic", "give a restart this wrote")
        length = struct.unpack("<Q", prefix[8:])[0]
        if not 0 < length <= HEADER_LIMIT_BYTES:
            _refuse("RESTART-ENVELOPE", f"{path} declares a {length}-byte header (the cap is {HEADER_LIMIT_BYTES})",
                    "give a restart this wrote")
        raw = f.read(length)
        if len(raw) != length:
            _refuse("RESTART-ENVELOPE", f"{path} holds {len(raw)} of the {length} header bytes it declares",
                    "give a complete restart")
        try:
            header = json.loads(raw.decode("utf-8"))
        except (UnicodeDecodeError, ValueError) as e:
            _refuse("RESTART-ENVELOPE", f"{path}'s header is not JSON ({e})", "give a restart this wrote")
        if not isinstance(header, dict) or not isinstance(header.get("contract"), dict):
            _refuse("RESTART-ENVELOPE", f"{path}'s header is not a restart header", "give a restart this wrote")
        contract = header["contract"]
        if header.get("contract_sha256") != hashlib.sha256(json.dumps(contract, sort_keys=True).encode()).hexdigest():
            _refuse("RESTART-CONTRACT", f"{path}'s contract does not match its recorded digest",
                    "the file is damaged; continue from another restart")
        if contract.get("profile") != PROFILE:
            _refuse("RESTART-PROFILE", f"{path} is a {contract.get('profile')!r} restart, not {PROFILE}",
                    "continue with the build that wrote it")
        payload = size - 16 - length
        if int(header.get("payload_nbytes", -1)) != payload:
            _refuse("RESTART-ENVELOPE", f"{path} holds {payload} payload bytes; its header declares "
                    f"{header.get('payload_nbytes')}", "give a complete restart")
        specs = {s["name"]: s for s in contract.get("array_specs", [])}
        arrays = {}
        for row in header.get("arrays", []):
            name = row["name"]
            spec = specs.get(name)
            if spec is None or spec.get("dtype") not in _DTYPES:
                _refuse("RESTART-CONTRACT", f"{name} has no array spec in {path}", "give a restart this wrote")
            dt = np.dtype(_DTYPES[spec["dtype"]])
            shape = tuple(int(v) for v in spec["shape"])
            if int(row["nbytes"]) != dt.itemsize * int(np.prod(shape, dtype=np.int64)):
                _refuse("RESTART-CONTRACT", f"{name} declares {row['nbytes']} bytes for shape {shape}",
                        "give a restart this wrote")
            f.seek(16 + length + int(row["offset"]))
            data = f.read(int(row["nbytes"]))
            if len(data) != int(row["nbytes"]) or hashlib.sha256(data).hexdigest() != row.get("sha256"):
                _refuse("RESTART-DIGEST", f"{name}'s bytes do not match the SHA-256 in {path}'s header",
                        "the file is damaged; continue from another restart")
            arrays[name] = np.frombuffer(data, dtype=dt).reshape(shape).astype(dt.newbyteorder("="))
    return header, arrays


def write_restart(path: str | os.PathLike, step) -> dict:
    """Write the carried arrays of a moist step (MoistLargeStep or
    NativeMoistLargeStep, after its queued work) and its step count and
    model time.  Returns the header."""
    import torch  # noqa: PLC0415

    s = step.s
    dev = s["u3d"].device
    torch.cuda.synchronize(dev)
    host = {n: s[n].detach().cpu().numpy() for n in CARRIED}
    base = {n: s[n].detach().cpu().numpy() for n in BASE_STATE}
    n_done = int(step.completed_steps)
    fields = {"magic": "CM1FCP1", "step": n_done, "model_time_s": float(np.float64(n_done) * np.float64(step.cfg.dt)),
              "config": config_record(step.cfg), "base_state_sha256": _digest(base, BASE_STATE)}
    return write_envelope(path, fields, host)


def resume(step, path: str | os.PathLike) -> dict:
    """Continue `step` (built on the same configuration from its initial
    state, so its base state is rebuilt) from the restart at `path`: check the
    configuration and the base state's digest, copy every carried array back
    into the step's device arrays and take its step count.  Returns the
    header."""
    import torch  # noqa: PLC0415

    header, arrays = read_envelope(path)
    want = config_record(step.cfg)
    got = header.get("config")
    if got != want:
        diff = sorted(k for k in set(want) | set(got or {}) if (got or {}).get(k) != want.get(k))
        _refuse("RESTART-CONFIG", f"the restart was written for another configuration (differs in {', '.join(diff)})",
                "continue on the configuration that wrote it")
    s = step.s
    base = {n: s[n].detach().cpu().numpy() for n in BASE_STATE}
    if header.get("base_state_sha256") != _digest(base, BASE_STATE):
        _refuse("RESTART-BASE-STATE", "the rebuilt base state differs from the one the restart was written on",
                "rebuild the step from the same sounding and geometry")
    missing = [n for n in CARRIED if n not in arrays]
    if missing:
        _refuse("RESTART-INVENTORY", f"the restart lacks {', '.join(missing)}", "give a restart this wrote")
    for n in CARRIED:
        t = s[n]
        a = arrays[n]
        if tuple(a.shape) != tuple(t.shape) or np.dtype(a.dtype) != np.dtype(str(t.dtype).replace("torch.", "")):
            _refuse("RESTART-INVENTORY", f"{n} is {a.dtype}{a.shape} in the restart and {t.dtype}{tuple(t.shape)} "
                    "in the step", "continue on the configuration that wrote it")
    torch.cuda.synchronize(s["u3d"].device)
    for n in CARRIED:
        s[n].copy_(torch.from_numpy(np.ascontiguousarray(arrays[n])))
    torch.cuda.synchronize(s["u3d"].device)
    step.completed_steps = int(header["step"])
    return header
