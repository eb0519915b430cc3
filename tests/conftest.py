"""Shared pytest configuration.

Tests marked ``gpu`` call the CUDA library through its C ABI and need a B200;
everything else runs on the CPU (oracle pins, host logic, ABI exports).
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture
def rng():
    return np.random.default_rng(12345)


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
        return {k: z[k] for k in z.files}
