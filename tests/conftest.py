import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "amr-lbm-openmp-2d_b200")
for p in (PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and the built libamrlbm.so")
    config.addinivalue_line("markers", "slow: long CPU-oracle runs")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the oracle and the library (no-ops when up to date)."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    subprocess.run(["make", "-s", "-C", PKG], check=True)
