"""Shared test setup: repo root on sys.path, the hyphenated package importable as `fe`,
and the `gpu` marker for tests that need a B200."""
from __future__ import annotations

import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def fe():
    return importlib.import_module("fasteddy-model_b200")


def interior(a):
    """Interior cells of a halo-inclusive field (last three axes)."""
    return a[..., 3:-3, 3:-3, 3:-3]


def rel_l2(a, b) -> float:
    import numpy as np

    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = float(np.linalg.norm(b.ravel()))
    d = float(np.linalg.norm((a - b).ravel()))
    return d / n if n > 0 else d
