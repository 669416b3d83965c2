"""Build libgm1b.so for sm_100a with nvcc (no GPU needed; nvcc cross-compiles).

    python -m gm1_b200.csrc.build [--verbose]

Flags: -gencode arch=compute_100a,code=sm_100a, -O3, -lineinfo and the
library's arithmetic contract --fmad=false -prec-div=true -prec-sqrt=true
-ftz=false (binary32 one operation at a time, as the reference kernels).
The library is written in-tree to gm1_b200/lib/libgm1b.so.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

CSRC = Path(__file__).resolve().parent
PKG = CSRC.parent
ROOT = PKG.parent
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libgm1b.so"
SOURCES = ("capi.cu", "periodic_lane.cu", "advection5.cu", "kessler.cu", "tke.cu", "scalar_rk.cu",
           "moist_bridge.cu", "initial_state.cu", "limits.cu", "closure.cu", "stress.cu", "stress_terrain.cu", "tke_evolution.cu", "momentum5.cu", "terrain_open.cu", "moist_step.cu", "vertical.cu", "moist_large_step.cu", "adjoint.cu", "selftest.cu")
ARCH = ("-gencode", "arch=compute_100a,code=sm_100a")
FLAGS = (
    "-O3", "-std=c++17", "-lineinfo",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-Xcompiler", "-ffp-contract=off",
    "--expt-relaxed-constexpr",
)


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return [CSRC / s for s in SOURCES]


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "gm1b.h"]
    return any(p.stat().st_mtime > t for p in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    objs = []
    build_dir = LIB_DIR / "_obj"
    build_dir.mkdir(exist_ok=True)
    for src in sources():
        obj = build_dir / (src.stem + ".o")
        cmd = [nvcc(), *ARCH, *FLAGS, "-I", str(ROOT / "include"), "-dc" if False else "-c", str(src), "-o", str(obj)]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    return LIB


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--verbose", action="store_true")
    p.add_argument("--ptxas-info", action="store_true")
    args = p.parse_args()
    out = build(args.verbose, args.ptxas_info)
    print(out)


if __name__ == "__main__":
    sys.exit(main())
