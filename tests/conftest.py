import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU-only checks")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the oracle and the native library in-tree once per session (incremental)."""
    import subprocess

    if not (REPO / "oracle" / "liboracle.so").exists() or os.environ.get("AUTAN_REBUILD"):
        subprocess.run(["make", "-s", "-C", str(REPO / "oracle")], check=True)
    lib = REPO / "autan_b200" / "_lib" / "libautan_b200.so"
    if not lib.exists() or os.environ.get("AUTAN_REBUILD"):
        from autan_b200 import build

        build.build()
    yield
