"""The short-path correctly rounded reciprocal of the column solves
(rcp_rn: hardware approximation plus one FMA Newton-Raphson step) gives
CUDA's __frcp_rn word on every one of the 2^32 binary32 inputs."""

from __future__ import annotations

import ctypes

import pytest
import torch

from gm1_b200 import _native

pytestmark = pytest.mark.gpu


def test_short_path_reciprocal_is_frcp_rn_on_every_word():
    lib = _native.lib()
    lib.gm1b_selftest_reciprocal.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.gm1b_selftest_reciprocal.restype = ctypes.c_int32
    counts = torch.zeros(2, dtype=torch.int64, device="cuda:0")
    first = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    stream = torch.cuda.current_stream()
    _native.check(lib.gm1b_selftest_reciprocal(counts.data_ptr(), first.data_ptr(),
                                               ctypes.c_void_p(stream.cuda_stream)), "gm1b_selftest_reciprocal")
    torch.cuda.synchronize()
    bad, fast = (int(v) for v in counts.cpu())
    word = int(first.cpu()[0]) & 0xFFFFFFFF
    assert fast > 3_000_000_000  # most words take the short path
    assert bad == 0, (bad, hex(word))
