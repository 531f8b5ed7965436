"""Shared fixtures. `-m gpu` tests need a CUDA device; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def dm():
    from dumato_b200 import build as _build

    _build.build()
    import dumato_b200

    return dumato_b200


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def gpu(dm):
    if dm.device_count() < 1:
        pytest.fail("no CUDA device visible to libdmb200 (gpu tests must run on a GPU box)")
    return True
