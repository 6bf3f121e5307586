import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Builds the oracle and the product library when they are missing (make is incremental)."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    if not os.path.exists(os.path.join(ROOT, "cells_b200", "libcells.so")):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "cells_b200", "csrc")], check=True)
    yield

