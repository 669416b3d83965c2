"""The allocation-free Kessler entry point gm1b_kessler_driver_static.

It exists for callers that cannot allocate device memory of their own (a
host model bound through the C ABI whose device memory belongs to another
runtime's pool, or a process whose device memory another framework reserves
up front) and so cannot hand gm1b_kessler_driver a workspace.  Its scratch is
a static device array shared by every call on a device.

The test drives both entry points through the C ABI on the same inputs for
two calls in a row (the second call starting from the first call's output).
Both run the same kernels in the same order on the same inputs, only with the
scratch at another address, so the static one must give the workspace one's
words exactly: every field, the budgets and the status words.  It also checks
that a grid too large for the static array is refused with a clear error.
This file is collected last so a failure here never hides another test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from gm1_b200.kessler import _bind, _KesslerArrays, create_cuda_gm1_kessler_driver_workspace
from tests.golden.make_golden import kessler_fixture

pytestmark = pytest.mark.gpu

NAMES = [n for n, _ in _KesslerArrays._fields_ if n not in ("satadj_iterations", "nfall")]


def _lib():
    lib = _bind()
    lib.gm1b_kessler_driver_static.argtypes = [ctypes.c_int32] * 3 + [
        ctypes.POINTER(_KesslerArrays), ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
        ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
    lib.gm1b_kessler_driver_static.restype = ctypes.c_int32
    return lib


def _device(host):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in host.items()}


def _struct(d):
    return _KesslerArrays(**{n: d[n].data_ptr() for n in NAMES})


def test_static_scratch_entry_matches_workspace_entry_on_two_calls():
    lib = _lib()
    ni, nj, nk, dz, dt = 96, 64, 40, 100.0, 20.0
    host = kessler_fixture(ni, nj, nk, dz, 123)
    with_ws = _device(host)
    static = _device(host)
    ws = create_cuda_gm1_kessler_driver_workspace(ni=ni, nj=nj, nk=nk)
    status = torch.full((2,), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    for call in range(2):
        s1 = _struct(with_ws)
        rc = lib.gm1b_kessler_driver(ni, nj, nk, ctypes.byref(s1), 1000.0, 1000.0, dz, dt, 2, 0,
                                     ctypes.c_void_p(ws.buffer.data_ptr()), ws.buffer.numel(),
                                     ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.gm1b_last_error()
        s2 = _struct(static)
        rc = lib.gm1b_kessler_driver_static(ni, nj, nk, ctypes.byref(s2), 1000.0, 1000.0, dz, dt, 2, 0,
                                            ctypes.c_void_p(status.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.gm1b_last_error()
        torch.cuda.synchronize()
        want = {k: v.cpu().numpy() for k, v in with_ws.items()}
        got = {k: v.cpu().numpy() for k, v in static.items()}
        for name in want:
            w, g = want[name], got[name]
            assert np.array_equal(w.view(np.uint8), g.view(np.uint8)), (call, name)
        assert status.cpu().tolist() == ws.status.cpu().tolist()[:2], call


def test_static_scratch_entry_refuses_oversize_grids():
    lib = _lib()
    s = _KesslerArrays()
    rc = lib.gm1b_kessler_driver_static(1024, 1024, 80, ctypes.byref(s), 1.0, 1.0, 1.0, 1.0, 2, 0, None, None)
    assert rc == -1
    assert b"static array" in lib.gm1b_last_error()
