import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path against the oracle")


@pytest.fixture(scope="session")
def built():
    """Build librmd.so and the oracle once per session."""
    from raymond_b200 import build as b
    import oracle_ctypes

    b.build()
    oracle_ctypes.build()
    return True


@pytest.fixture(scope="session")
def gpu_ctx(built):
    from raymond_b200 import api

    return api.Context(0)
