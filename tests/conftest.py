"""Shared fixtures.  `-m gpu` tests need a CUDA device and the in-tree build."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_built():
    from egg_b200 import build

    build.build()


_ensure_built()


def gpu_available() -> bool:
    from egg_b200 import cpp_core

    return cpp_core.device_count() > 0


@pytest.fixture(scope="session")
def core():
    from egg_b200 import cpp_core

    return cpp_core


@pytest.fixture(scope="session")
def gpu(core):
    if core.device_count() == 0:
        pytest.fail("GPU test selected but no CUDA device is visible")
    return core


GOLDEN = ROOT / "tests" / "golden"
