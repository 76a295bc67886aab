"""Shared test setup: the `gpu` marker, import paths and seeded inputs."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "quarry-gpu_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def rng():
    return np.random.default_rng(1234)


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def cuda():
    if not gpu_available():
        pytest.fail("GPU test collected on a host without a CUDA device")
    import torch

    torch.cuda.init()
    return torch
