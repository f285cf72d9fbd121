"""Shared test setup: the `gpu` marker, library builds, and grid helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the oracle and the engine library if they are missing or stale."""
    import oracle
    from openems_b200 import build as engine_build
    oracle.build()
    if engine_build.needs_build():
        engine_build.build()


def rel_l2(a, b):
    """||a - b|| / ||b|| in f64 (0 when both are zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    if den == 0.0:
        return 0.0 if num == 0.0 else np.inf
    return num / den
