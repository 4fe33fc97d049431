import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the oracle (test infrastructure) and the product library in-tree."""
    from oracle import build as oracle_build
    oracle_build.build()
    from mutracer_b200 import build as product_build
    product_build.build()
    from oracle import ref_hosts
    ref_hosts.build()
    yield


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
