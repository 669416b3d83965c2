"""Golden vectors from the reference's own CUDA kernel texts, run on the host.

Several operators of the reference exist only as CUDA C text inside its
Python modules (no NumPy twin): the flat stretched-column closure among them
(src/cm1core/cuda_gm1_flat_stretched_closure.py).  Their texts use only
binary32 add/subtract/multiply/divide intrinsics (__fadd_rn, __fsub_rn,
__fmul_rn, __fdiv_rn), binary64 WENO weights and integer indexing, so a
C++ compiler on the host reproduces the device words exactly once those
intrinsics are plain IEEE operations (no contraction: -ffp-contract=off).
This script imports the reference (read only, never copied into the
repository), writes each text beside a small header that supplies the
intrinsics and a launch index, compiles it with g++ into a temporary
directory, runs its kernels one thread index at a time in their launch
order, and stores whole input/output array sets as .npz fixtures here.

    python tests/golden/make_kernel_text_golden.py --reference /path/to/gm1 flat-closure
    python tests/golden/make_kernel_text_golden.py --reference /path/to/gm1 flat-stress

The fixtures pin the oracle restatements (tests/test_oracle_flat_closure.py)
and through them the CUDA kernels.
"""

from __future__ import annotations

import argparse
import ctypes
import re
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

HOST_HEADER = r"""
#include <cmath>
#include <cstdint>
struct gm1_host_dim3 { unsigned x, y, z; };
static gm1_host_dim3 blockIdx = {0u, 0u, 0u}, threadIdx = {0u, 0u, 0u};
static gm1_host_dim3 blockDim = {1u, 1u, 1u}, gridDim = {1u, 1u, 1u};
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
static inline float __fadd_rn(float a, float b) { return a + b; }
static inline float __fsub_rn(float a, float b) { return a - b; }
static inline float __fmul_rn(float a, float b) { return a * b; }
static inline float __fdiv_rn(float a, float b) { return a / b; }
extern "C" void gm1_host_launch_index(unsigned block, unsigned thread, unsigned block_dim, unsigned grid_dim) {
  blockIdx.x = block; threadIdx.x = thread; blockDim.x = block_dim; gridDim.x = grid_dim;
}
"""

_CTYPE = {"float": ctypes.c_float, "double": ctypes.c_double, "unsigned": ctypes.c_uint, "int": ctypes.c_int,
          "unsigned long long": ctypes.c_ulonglong}


class HostKernels:
    """The kernels of one reference CUDA text, compiled for the host."""

    def __init__(self, text: str, workdir: Path, name: str) -> None:
        src = workdir / f"{name}.cpp"
        src.write_text(HOST_HEADER + "\n" + text)
        lib = workdir / f"lib{name}.so"
        subprocess.run(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                        "-w", str(src), "-o", str(lib)], check=True)
        self.lib = ctypes.CDLL(str(lib))
        self.lib.gm1_host_launch_index.argtypes = [ctypes.c_uint] * 4
        self.signatures = {}
        for m in re.finditer(r'extern "C" __global__ void (\w+)\(([^)]*)\)', text):
            types = []
            for p in m.group(2).split(","):
                p = p.strip()
                if "*" in p:
                    types.append(ctypes.c_void_p)
                    continue
                base = p.rsplit(" ", 1)[0].replace("const ", "").strip()
                types.append(_CTYPE[base])
            self.signatures[m.group(1)] = types
            fn = getattr(self.lib, m.group(1))
            fn.argtypes = types
            fn.restype = None

    @staticmethod
    def _arg(x):
        return x.ctypes.data if isinstance(x, np.ndarray) else x

    def grid_stride(self, name: str, *args) -> None:
        """A grid-stride kernel: one host thread covers every index."""
        self.lib.gm1_host_launch_index(0, 0, 1, 1)
        getattr(self.lib, name)(*(self._arg(a) for a in args))

    def per_thread(self, name: str, threads: int, *args) -> None:
        """A one-index-per-thread kernel over thread indices 0..threads-1."""
        fn = getattr(self.lib, name)
        conv = [self._arg(a) for a in args]
        for t in range(threads):
            self.lib.gm1_host_launch_index(t, 0, 1, threads)
            fn(*conv)


def f32(x) -> np.ndarray:
    return np.ascontiguousarray(x, dtype=np.float32)


# ---------------------------------------------------------------------------
# flat stretched-column closure: calcdef, turbt, TKE advw
# ---------------------------------------------------------------------------
def flat_closure_fixture(ni: int, nj: int, nk: int, seed: int) -> dict[str, np.ndarray]:
    """Inputs of the flat closure texts on a stretched column (20 m at the
    ground to 200 m aloft): winds with both signs, positive densities with
    horizontal structure, TKE and mixing coefficients, padded mass fluxes
    and the column metrics of the generated coordinate."""
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle import vertical as ov

    spec = {10: (1100.0, 40.0, 700.0), 14: (1630.0, 40.0, 1030.0), 12: (1400.0, 40.0, 900.0)}[nk]
    rc, lv = ov.vertical_levels(1, nk, 100.0, spec[0], spec[1], spec[2], 20.0, 200.0)
    assert rc == 0
    rng = np.random.default_rng(seed)
    mass, face = (nk, nj, ni), (nk + 1, nj, ni)
    a = {
        "u3d": rng.uniform(-12.0, 14.0, (nk, nj, ni + 1)), "v3d": rng.uniform(-11.0, 9.0, (nk, nj + 1, ni)),
        "w3d": rng.uniform(-3.0, 4.0, face),
        "rho": 1.1 + 0.05 * rng.standard_normal(mass), "rf": 1.1 + 0.05 * rng.standard_normal(face),
        "kmh": rng.uniform(0.0, 40.0, face), "kmv": rng.uniform(0.0, 30.0, face),
        "tke3d": rng.uniform(0.0, 2.0, face), "tkea": rng.uniform(0.0, 2.0, face),
        "tketen": rng.uniform(-1e-3, 1e-3, face), "divx": rng.uniform(-1e-3, 1e-3, mass),
        "rru": rng.uniform(-15.0, 15.0, (nk + 2, nj + 6, ni + 7)), "rrv": rng.uniform(-15.0, 15.0, (nk + 2, nj + 7, ni + 6)),
        "rrw": rng.uniform(-3.0, 3.0, (nk + 3, nj + 6, ni + 6)),
    }
    a["tke3d"][0] = a["tke3d"][nk] = 0.0
    # the two open-boundary branches of every flux and a few tiny TKE words
    a["tke3d"][2, 1, :3] = 1e-11
    mhp, mfp = np.asarray(lv["mh"], np.float32), np.asarray(lv["mf"], np.float32)
    a["mh_profile"], a["mf_profile"] = mhp, mfp
    a["mh"] = np.broadcast_to(mhp[1:nk + 1, None, None], mass)
    a["mf"] = np.broadcast_to(mfp[1:nk + 2, None, None], face)
    zh, zf = np.asarray(lv["zh"], np.float32), np.asarray(lv["zf"], np.float32)
    c2 = np.empty(nk + 1, np.float32)
    for k in range(1, nk + 2):
        c2[k - 1] = (zf[k] - zh[k - 1]) / (zh[k] - zh[k - 1])
    a["c2"] = np.broadcast_to(c2[:, None, None], face)
    a["c1"] = np.broadcast_to((np.float32(1.0) - c2)[:, None, None], face)
    a["rrf0"] = np.broadcast_to((1.0 / (1.05 + 0.01 * np.arange(nk + 1)))[:, None, None], face)
    out = {k: f32(v) for k, v in a.items()}
    out["rdz"] = np.float32(np.float32(1.0) / np.float32(100.0))
    return out


def make_flat_closure(reference: Path) -> None:
    sys.path.insert(0, str(reference / "src"))
    import cm1core.cuda_gm1_flat_stretched_closure as fc

    grids = ((12, 10, 10, 11), (9, 13, 14, 12))
    with tempfile.TemporaryDirectory() as tmp:
        work = Path(tmp)
        closure = HostKernels(fc.flat_stretched_closure_source(max_nk=64), work, "flat_closure")
        tke = HostKernels(fc.GM1_FLAT_STRETCHED_TKE_ADVECTION_SOURCE, work, "flat_tke")
        for ni, nj, nk, seed in grids:
            a = flat_closure_fixture(ni, nj, nk, seed)
            dx, dy, dt = 450.0, 520.0, 2.0
            rdx, rdy = np.float32(np.float32(1.0) / np.float32(dx)), np.float32(np.float32(1.0) / np.float32(dy))
            rdz = float(a["rdz"])
            u = np.uint32
            out: dict[str, np.ndarray] = {}
            # calcdef (turb.F:4766-5388): zero fill, mass, face, reduce
            s11, s22, s33 = (np.zeros((nk, nj, ni), np.float32) for _ in range(3))
            s12 = np.zeros((nk, nj + 1, ni + 1), np.float32)
            s13 = np.zeros((nk + 1, nj, ni + 1), np.float32)
            s23 = np.zeros((nk + 1, nj + 1, ni), np.float32)
            defv, defh = np.zeros((nk + 1, nj, ni), np.float32), np.zeros((nk + 1, nj, ni), np.float32)
            closure.grid_stride("gm1_flat_calcdef_mass_v1", a["u3d"], a["v3d"], a["w3d"], a["rho"], a["mh_profile"],
                                s11, s22, s33, s12, u(ni), u(nj), u(nk), float(rdx), float(rdy), rdz)
            closure.grid_stride("gm1_flat_calcdef_face_v1", a["u3d"], a["v3d"], a["w3d"], a["rf"], a["mf"], s13, s23,
                                u(ni), u(nj), u(nk), float(rdx), float(rdy), rdz)
            closure.grid_stride("gm1_flat_calcdef_reduce_v1", a["rf"], a["c1"], a["c2"], s11, s22, s33, s12, s13, s23,
                                defv, defh, u(ni), u(nj), u(nk))
            out["defv"], out["defh"] = defv, defh
            # turbt on tke3d into a copy of tketen
            ten = a["tketen"].copy()
            closure.per_thread("gm1_flat_turbt_v1", ni * nj, a["tke3d"], a["kmh"], a["kmv"], a["rho"], a["rf"],
                               a["mh"], a["mf"], ten, u(ni), u(nj), u(nk), float(rdx), float(rdy), rdz, dt)
            out["tketen_turbt"] = ten
            # the three RK stages from tke3d (CartesianClosure.tke_rk,
            # cuda_cartesian_closure.py:1635-1685) on tketen after turbt
            cur = a["tke3d"].copy()
            weps = float(np.float32(np.float32(100.0) * np.float32(1e-18)))
            for nrk in (1, 2, 3):
                nxt = np.zeros_like(cur)
                dttmp = float(np.float32(np.float32(dt) / np.float32(4 - nrk)))
                tke.per_thread("gm1_flat_tke_advw_rk_v1", (nk + 1) * nj * ni, cur, a["tkea"], ten, a["c1"], a["c2"],
                               a["rrf0"], a["rru"], a["rrv"], a["rrw"], a["divx"], nxt, u(ni), u(nj), u(nk), u(3),
                               dx, dy, dttmp, u(1 if nrk == 3 else 0), weps, a["mf_profile"], rdz)
                out[f"tke_stage{nrk}"] = nxt
                cur = nxt
            meta = np.array([ni, nj, nk], np.int32)
            path = HERE / f"flat_closure_{ni}x{nj}x{nk}.npz"
            np.savez_compressed(path, meta=meta, dx=np.float32(dx), dy=np.float32(dy), dt=np.float32(dt),
                                **{f"in_{k}": v for k, v in a.items()}, **{f"out_{k}": v for k, v in out.items()})
            print("wrote", path.name)


# ---------------------------------------------------------------------------
# flat stretched-column held closure: gettau, turbu/turbv/turbw, turbs
# ---------------------------------------------------------------------------
def make_flat_stress(reference: Path) -> None:
    """The strain passes, gettau (enqueue_flat_gettau), the momentum stress
    (enqueue_flat_momentum_stress, two_part=None) and the flat turbs of theta
    and three moisture rows (the pad/pack texts of
    cuda_gm1_scalar_turbulence.py, then gm1_flat_turbs_xy_flux_v1 and
    gm1_flat_turbs_implicit_apply_v1 with iflux = 0) on the flat closure's
    fixtures, in the closure's launch order."""
    sys.path.insert(0, str(reference / "src"))
    import cm1core.cuda_gm1_flat_stretched_closure as fc
    import cm1core.cuda_gm1_scalar_turbulence as st

    grids = ((12, 10, 10, 21), (9, 13, 14, 22))
    with tempfile.TemporaryDirectory() as tmp:
        work = Path(tmp)
        closure = HostKernels(fc.flat_stretched_closure_source(max_nk=64), work, "flat_closure")
        scalar = HostKernels(st.CUDA_GM1_SCALAR_TURBULENCE_SOURCE, work, "scalar_turbulence")
        for ni, nj, nk, seed in grids:
            a = flat_closure_fixture(ni, nj, nk, seed)
            rng = np.random.default_rng(seed + 100)
            mass, face = (nk, nj, ni), (nk + 1, nj, ni)
            a["rr"] = f32(np.float32(1.0) / a["rho"])
            a["khh"] = f32(rng.uniform(0.0, 60.0, face))
            a["khv"] = f32(rng.uniform(0.0, 60.0, face))
            a["th0"] = f32(np.linspace(300.0, 330.0, nk))
            a["tha"] = f32(rng.normal(0.0, 1.5, mass))
            a["qa"] = f32(np.abs(rng.normal(0.0, 4e-3, (6, nk, nj, ni))))
            for n, sh in (("uten", (nk, nj, ni + 1)), ("vten", (nk, nj + 1, ni)), ("wten", face)):
                a[n] = f32(rng.normal(0.0, 1e-3, sh))
            a["thten1"] = f32(rng.normal(0.0, 1e-4, mass))
            a["qten"] = f32(rng.normal(0.0, 1e-7, (6, nk, nj, ni)))
            dx, dy, dt = 450.0, 520.0, 2.0
            rdx, rdy = np.float32(np.float32(1.0) / np.float32(dx)), np.float32(np.float32(1.0) / np.float32(dy))
            rdz = float(a["rdz"])
            u = np.uint32
            dims = (u(ni), u(nj), u(nk))
            out: dict[str, np.ndarray] = {}
            s11, s22, s33 = (np.zeros(mass, np.float32) for _ in range(3))
            s12 = np.zeros((nk, nj + 1, ni + 1), np.float32)
            s13 = np.zeros((nk + 1, nj, ni + 1), np.float32)
            s23 = np.zeros((nk + 1, nj + 1, ni), np.float32)
            closure.grid_stride("gm1_flat_calcdef_mass_v1", a["u3d"], a["v3d"], a["w3d"], a["rho"], a["mh_profile"],
                                s11, s22, s33, s12, *dims, float(rdx), float(rdy), rdz)
            closure.grid_stride("gm1_flat_calcdef_face_v1", a["u3d"], a["v3d"], a["w3d"], a["rf"], a["mf"], s13, s23,
                                *dims, float(rdx), float(rdy), rdz)
            out.update(s11=s11, s22=s22, s33=s33, s12=s12, s13=s13, s23=s23)
            t11, t22, t33 = (np.zeros(mass, np.float32) for _ in range(3))
            t12 = np.zeros((nk, nj + 1, ni + 1), np.float32)
            t13 = np.zeros((nk + 1, nj, ni + 1), np.float32)
            t23 = np.zeros((nk + 1, nj + 1, ni), np.float32)
            closure.grid_stride("gm1_flat_gettau_normal_v1", s11, s22, s33, a["kmh"], t11, t22, t33, *dims)
            closure.grid_stride("gm1_flat_gettau_t12_v1", s12, a["kmh"], t12, *dims)
            closure.grid_stride("gm1_flat_gettau_t13_v1", s13, a["kmv"], t13, *dims)
            closure.grid_stride("gm1_flat_gettau_t23_v1", s23, a["kmv"], t23, *dims)
            out.update(t11=t11, t22=t22, t33=t33, t12=t12, t13=t13, t23=t23)
            uten, vten, wten = a["uten"].copy(), a["vten"].copy(), a["wten"].copy()
            common = (a["kmv"], a["rho"], a["rf"], a["mh"], a["mf"], a["mh_profile"])
            closure.per_thread("gm1_flat_turbu_v1", nj * (ni + 1), t11, t12, t13, *common, a["u3d"], a["w3d"], uten,
                               a["mh_profile"], uten, *dims, float(rdx), float(rdy), rdz, dt, u(0))
            closure.per_thread("gm1_flat_turbv_v1", (nj + 1) * ni, t12, t22, t23, *common, a["v3d"], a["w3d"], vten,
                               a["mh_profile"], vten, *dims, float(rdx), float(rdy), rdz, dt, u(0))
            closure.per_thread("gm1_flat_turbw_v1", nj * ni, t13, t23, t33, a["kmh"], a["rho"], a["rf"], a["mh"],
                               a["mf"], a["w3d"], wten, *dims, float(rdx), float(rdy), rdz, dt)
            out.update(uten=uten, vten=vten, wten=wten)
            # turbs: theta then qv, qc, qr (solve1.F:1169-1233), dz the
            # coordinate's reference spacing, no surface flux
            hx, hy = ni + 2, nj + 2
            rhoh = np.zeros((nk, hy, hx), np.float32)
            khhh = np.zeros((nk + 1, hy, hx), np.float32)
            gzh, rgzh = np.zeros((hy, hx), np.float32), np.zeros((hy, hx), np.float32)
            ones = np.ones((nj, ni), np.float32)
            scalar.grid_stride("gm1_turbs_pad_static_open_v1", a["rho"], a["khh"], ones, ones, rhoh, khhh, gzh, rgzh,
                               *dims)
            thten1, qten = a["thten1"].copy(), a["qten"].copy()
            fx = np.zeros((nk, nj, ni + 1), np.float32)
            fy = np.zeros((nk, nj + 1, ni), np.float32)
            cp, dp = np.zeros(mass, np.float32), np.zeros(mass, np.float32)
            sflux = np.zeros((nj, ni), np.float32)
            dz = float(np.float32(1.0) / np.float32(rdz))
            for species, target in ((0xFFFFFFFF, thten1), (0, qten[0]), (1, qten[1]), (2, qten[2])):
                sh = np.zeros((nk, hy, hx), np.float32)
                scalar.grid_stride("gm1_turbs_pack_scalar_open_v1", a["th0"], a["tha"], a["qa"], sh, *dims,
                                   u(species))
                closure.grid_stride("gm1_flat_turbs_xy_flux_v1", sh, rhoh, khhh, fx, fy, *dims, dx, dy)
                closure.per_thread("gm1_flat_turbs_implicit_apply_v1", ni * nj, sh, a["rho"], a["rr"], a["rf"],
                                   a["mh"], a["mf"], a["khv"], fx, fy, sflux, cp, dp, target, *dims, dx, dy, dz, dt,
                                   u(0))
            out.update(thten1=thten1, qten=qten)
            path = HERE / f"flat_stress_{ni}x{nj}x{nk}.npz"
            np.savez_compressed(path, meta=np.array([ni, nj, nk], np.int32), dx=np.float32(dx), dy=np.float32(dy),
                                dt=np.float32(dt), dz=np.float32(dz), **{f"in_{k}": v for k, v in a.items()},
                                **{f"out_{k}": v for k, v in out.items()})
            print("wrote", path.name)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True)
    ap.add_argument("what", choices=["flat-closure", "flat-stress"])
    args = ap.parse_args()
    if args.what == "flat-closure":
        make_flat_closure(args.reference)
    elif args.what == "flat-stress":
        make_flat_stress(args.reference)


if __name__ == "__main__":
    main()
