"""The FP64 run of the oracle's composed moist step - TEST INFRASTRUCTURE ONLY.

The oracle's composition (oracle.moist_composition.OracleMoistStep) evaluated
with every binary32 operation in binary64: liboracle_gm1_f64.so is the same C
source built with -DORACLE_F64 (oracle/real.h), so it runs the same operators
in the same order and differs from the binary32 oracle only by rounding.  Its
fields, started from the same float32 words as a float32 run, are the
reference each float32 run's rounding error is measured against.

The working precision is fixed per process (oracle.periodic reads
GM1B_ORACLE_REAL at import), so the run happens in a child process:

    run_fp64(cfg, state, metrics, steps, snapshots) -> {step: {field: float64}}

and the child's entry point is ``python -m oracle.fp64_twin IN OUT``.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path
from types import SimpleNamespace

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
CFG_KEYS = ("ni", "nj", "nk", "dx", "dy", "dz", "dt", "nsound", "alph", "kdiv", "lateral_sides", "obc")
# the prognostic words a step leaves (the state names the tests compare)
OUT_FIELDS = ("u3d", "v3d", "w3d", "th3d", "pp3d", "q3d", "tke3d")


def _cfg_dict(cfg) -> dict:
    d = {k: getattr(cfg, k) for k in CFG_KEYS}
    d["lateral_sides"] = list(d["lateral_sides"])
    d["stretched"] = getattr(cfg, "column", None) is not None
    d["apmasscon"] = bool(getattr(cfg, "apmasscon", True))
    d["sgs_diffusion"] = bool(getattr(cfg, "sgs_diffusion", False))
    d["rayleigh"] = bool(getattr(cfg, "rayleigh", False))
    d["dissipative_heating"] = bool(getattr(cfg, "dissipative_heating", False))
    d["rayleigh_zd_m"] = float(getattr(cfg, "rayleigh_zd_m", 15000.0))
    d["rayleigh_rdalpha"] = float(getattr(cfg, "rayleigh_rdalpha", 3.3333333333e-3))
    return d


def run_fp64(cfg, state: dict, metrics: dict, steps: int, snapshots=None, threads: int | None = None) -> dict:
    """Step the binary64 composition `steps` times from the given float32
    starting state (host numpy arrays); return {step: {name: float64 array}}
    for each step in `snapshots` (default: the last)."""
    snaps = sorted(set(snapshots or [steps]))
    if not snaps or snaps[0] < 1 or snaps[-1] > steps:
        raise ValueError("snapshots must lie in 1..steps")
    with tempfile.TemporaryDirectory() as d:
        src, dst = Path(d) / "in.npz", Path(d) / "out.npz"
        arrays = {f"s:{k}": np.asarray(v) for k, v in state.items()}
        arrays.update({f"m:{k}": np.asarray(v) for k, v in metrics.items()})
        np.savez(src, **arrays)
        job = {"cfg": _cfg_dict(cfg), "steps": int(steps), "snapshots": snaps, "threads": threads}
        env = dict(os.environ, GM1B_ORACLE_REAL="f64")
        env["PYTHONPATH"] = str(ROOT) + (os.pathsep + env["PYTHONPATH"] if env.get("PYTHONPATH") else "")
        subprocess.run([sys.executable, "-m", "oracle.fp64_twin", str(src), str(dst), json.dumps(job)],
                       env=env, cwd=str(ROOT), check=True)
        with np.load(dst) as z:
            out: dict[int, dict[str, np.ndarray]] = {}
            for key in z.files:
                step, name = key.split(":", 1)
                out.setdefault(int(step), {})[name] = z[key]
    return out


def _child(src: str, dst: str, job: dict) -> None:
    from oracle import periodic as orc  # noqa: PLC0415
    from oracle.moist_composition import OracleMoistStep  # noqa: PLC0415

    if not orc.F64:
        raise RuntimeError("the FP64 run needs GM1B_ORACLE_REAL=f64")
    if job.get("threads"):
        orc.set_threads(int(job["threads"]))
    state, metrics = {}, {}
    with np.load(src) as z:
        for key in z.files:
            kind, name = key.split(":", 1)
            a = z[key]
            if a.dtype == np.float32:  # the same words, widened exactly
                a = a.astype(np.float64)
            (state if kind == "s" else metrics)[name] = np.ascontiguousarray(a)
    c = dict(job["cfg"])
    stretched = c.pop("stretched")
    c["lateral_sides"] = tuple(c["lateral_sides"])
    cfg = SimpleNamespace(**c, column=SimpleNamespace() if stretched else None)
    step = OracleMoistStep(cfg, state, metrics)
    out = {}
    for n in range(1, int(job["steps"]) + 1):
        step.step()
        if n in job["snapshots"]:
            for name in OUT_FIELDS:
                out[f"{n}:{name}"] = np.array(state[name], dtype=np.float64)
    np.savez(dst, **out)


if __name__ == "__main__":
    _child(sys.argv[1], sys.argv[2], json.loads(sys.argv[3]))
