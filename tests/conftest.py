"""Shared fixtures: marker registration and in-tree builds of both libraries."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def wt_lib():
    """libwt.so, built in-tree if the sources changed (nvcc cross-compiles without a GPU)."""
    from windtunnel_b200 import _lib, build
    if os.environ.get("WT_SKIP_BUILD") != "1":
        build.build()
    return _lib.lib()
