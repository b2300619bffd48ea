"""Shared test setup: GPU marker, package import alias, golden fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "mbd-icenav_b200"))
import _pkg  # noqa: E402

_pkg.load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden64():
    return np.load(os.path.join(GOLDEN, "golden_f64.npz"))


@pytest.fixture(scope="session")
def golden32():
    return np.load(os.path.join(GOLDEN, "golden_f32.npz"))
