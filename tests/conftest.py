"""Shared pytest set-up: the ``gpu`` marker and fixture loaders."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / name, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def golden_kernels():
    return load_golden("kernels_small.npz")


@pytest.fixture(scope="session")
def golden_config1():
    return load_golden("config1.npz")


@pytest.fixture(scope="session")
def golden_sphere():
    return load_golden("sphere.npz")


@pytest.fixture(scope="session")
def golden_fiber():
    return load_golden("fiber_ops.npz")


def rel_err(a, b) -> float:
    """max |a - b| / max |b| (norm-wise relative error)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    if a.shape != b.shape:
        raise AssertionError(f"shape mismatch {a.shape} vs {b.shape}")
    den = np.max(np.abs(b)) if b.size else 0.0
    if den == 0.0:
        return float(np.max(np.abs(a))) if a.size else 0.0
    return float(np.max(np.abs(a - b)) / den)
