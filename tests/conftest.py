import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the engine's kernels)")


def close(a, b, tol):
    """The reference tests' tolerance: |a - b| <= tol (1 + max(|a|, |b|)) (kernel.rs:178-180)."""
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return np.abs(a - b) <= tol * (1.0 + np.maximum(np.abs(a), np.abs(b)))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o

    o.build()
    return o
