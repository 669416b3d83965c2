"""CM1's upper Rayleigh damping (irdamp = 1) on B200: the static damping
coefficients of the column and the held u, v, w and theta tendencies.

Drop-in mirror of the reference operator API (torch CUDA tensors in place of
CuPy arrays; the same array names and shapes):

  build_rayleigh_coefficients  cpu_build_rayleigh_coefficients
                               src/cm1core/cuda_rayleigh_held.py:264-383
                               (CM1 param.F:8631-8673) - host set-up, as there
  rayleigh_held_shapes,
  launch_cuda_rayleigh_held    src/cm1core/cuda_rayleigh_held.py:143, :523
                               (CM1 solve1.F:412-454)

The coefficients are formed once on the host in binary32 with the host's
float32 cosine (numpy), as the reference's builder forms them; the held
tendencies are a CUDA kernel (csrc/stress.cu, gm1b_rayleigh_held).
"""

from __future__ import annotations

import ctypes
import math
from typing import Any, Mapping

import numpy as np
import torch

from . import _native
from .closure import _require
from .periodic import CudaLaunch

# the supercell namelist's damping (irdamp = 1, rdalpha = 1/300 s^-1 above
# zd = 15 km)
SUPERCELL_RDALPHA = 3.3333333333e-3
SUPERCELL_ZD_M = 15000.0

ARRAY_NAMES = ("tauh", "taus", "tauf", "u0", "v0", "ua", "va", "wa", "tha", "uten1", "vten1", "wten1", "thten1")


class _Arrays(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ARRAY_NAMES]


def build_rayleigh_coefficients(zh, zf, *, damping_start_m: float) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(tauh, taus, tauf) of CM1 param.F's irdamp = 1 branch on heights zh
    (mass points) and zf (faces; the last one is the model top), any shape
    with zf one level longer: 0 at or below the damping start, else
    0.5*(1 - cos(pi*(z - start)/(top - start))), binary32 throughout with
    numpy's float32 cosine (the reference's builder's words)."""
    f = np.float32
    zh = np.ascontiguousarray(zh, f)
    zf = np.ascontiguousarray(zf, f)
    if zf.shape[0] != zh.shape[0] + 1 or zf.shape[1:] != zh.shape[1:]:
        raise ValueError("zf must hold one more level than zh")
    start, pi, half, one = f(damping_start_m), f(math.pi), f(0.5), f(1.0)
    top = zf[-1]

    def coefficient(height):
        out = np.zeros_like(height, dtype=f)
        mask = height > start
        numerator = np.subtract(height, start, dtype=f)
        denominator = np.subtract(top[None], start, dtype=f)
        angle = np.multiply(pi, np.divide(numerator, denominator, dtype=f), dtype=f)
        cosine = np.cos(angle, dtype=f)
        computed = np.multiply(half, np.subtract(one, cosine, dtype=f), dtype=f)
        out[mask] = computed[mask]
        return np.ascontiguousarray(out)

    tauh = coefficient(zh)
    return tauh, tauh.copy(), coefficient(zf)


def rayleigh_held_shapes(ni: int, nj: int, nk: int, *, profiles: bool = False) -> dict[str, tuple[int, ...]]:
    mass = (nk, nj, ni)
    if profiles:
        tau = {"tauh": (nk,), "taus": (nk,), "tauf": (nk + 1,)}
    else:
        tau = {"tauh": (nk, nj + 2, ni + 2), "taus": (nk, nj + 2, ni + 2), "tauf": (nk + 1, nj + 2, ni + 2)}
    return {**tau, "u0": (nk,), "v0": (nk,), "ua": (nk, nj, ni + 1), "va": (nk, nj + 1, ni), "wa": mass,
            "tha": mass, "uten1": (nk, nj, ni + 1), "vten1": (nk, nj + 1, ni), "wten1": mass, "thten1": mass}


def launch_cuda_rayleigh_held(arrays: Mapping[str, Any], *, ni: int, nj: int, nk: int,
                              rdalpha: float = SUPERCELL_RDALPHA, profiles: bool = False,
                              add_momentum: bool = False, stream: Any | None = None) -> CudaLaunch:
    """The held upper-damping tendencies (launch_cuda_rayleigh_held):
    uten1/vten1/wten1/thten1 assigned, or with ``add_momentum`` the momentum
    damping added into uten1/vten1/wten1 (the closure's held sum) and thten1
    assigned.  ``profiles``: tauh/taus/tauf are column profiles instead of
    one-halo 3-D arrays.  ``wa`` may be the first nk faces of a w array."""
    for name, value in (("ni", ni), ("nj", nj), ("nk", nk)):
        if isinstance(value, bool) or not isinstance(value, int) or value < 1:
            raise ValueError(f"{name} must be a positive integer")
    if isinstance(rdalpha, bool) or not isinstance(rdalpha, (int, float)) or not math.isfinite(rdalpha) \
            or rdalpha < 0.0:
        raise ValueError("rdalpha must be finite and >= 0")
    shapes = rayleigh_held_shapes(ni, nj, nk, profiles=profiles)
    a = _require(arrays, ARRAY_NAMES, shapes, "rayleigh-held")
    s = _Arrays(**{n: a[n].data_ptr() for n in ARRAY_NAMES})
    lib = _native.lib()
    if not getattr(lib, "_rayleigh_bound", False):
        i32 = ctypes.c_int32
        lib.gm1b_rayleigh_held.argtypes = [i32, i32, i32, ctypes.POINTER(_Arrays), i32, i32, ctypes.c_float,
                                           ctypes.c_void_p]
        lib.gm1b_rayleigh_held.restype = i32
        lib._rayleigh_bound = True
    device = a["uten1"].device
    st = torch.cuda.current_stream(device) if stream is None else stream
    with torch.cuda.device(device):
        _native.check(lib.gm1b_rayleigh_held(ni, nj, nk, ctypes.byref(s), 1 if profiles else 0,
                                             1 if add_momentum else 0, float(np.float32(rdalpha)),
                                             ctypes.c_void_p(st.cuda_stream)), "gm1b_rayleigh_held")
        ev = torch.cuda.Event()
        ev.record(st)
    return CudaLaunch(ev, {"operator": "rayleigh-held", "cell_words": ni * nj * nk})
