"""Shared test set-up: import paths, the ``gpu`` marker."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "jax-rans_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: long-running")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not gpu_available():
        pytest.skip("no CUDA device")
    return True


@pytest.fixture(scope="session", autouse=True)
def fresh_library(request):
    """The C-ABI library rebuilt in place when a source is newer (nvcc is on the GPU box too)."""
    if any(item.get_closest_marker("gpu") for item in request.session.items) and gpu_available():
        from jaxrans_b200.build import build
        build()
