import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "latticeboltzmannmethod-fonnesu-grassi-guffanti_b200")
for p in (HERE, os.path.join(PKG, "python")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running CPU reference comparison")


@pytest.fixture(scope="session")
def cuda_lib():
    """The in-tree CUDA library; GPU tests fail loudly if it cannot be loaded."""
    import llalbm_cuda

    return llalbm_cuda.lib()
