"""Shared test configuration.

Tests marked ``gpu`` need a CUDA device and the built libgm1b.so; everything
else runs on CPU.  The repository root is put on sys.path so ``gm1_b200`` and
the test-only ``oracle`` package import without installation.
"""

from __future__ import annotations

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")
