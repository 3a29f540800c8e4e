import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the kernels through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle and the CUDA library in-tree once per session."""
    from peridigm_b200.build import build

    build()
