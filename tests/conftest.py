"""Test configuration: the ``gpu`` marker and shared fixtures.

Tests marked ``gpu`` need a B200 (CUDA) and call the library through its C ABI; everything
else runs on the CPU (oracle vs golden vectors, host-side logic, library symbols).
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(GOLDEN / name))

    return load
