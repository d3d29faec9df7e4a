import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (the CUDA engine's parity and property tests)")


@pytest.fixture(scope="session")
def gpu_executor():
    """The native `cuda` stack; fails loudly when the native build or the GPU is missing."""
    import bohrium_b200 as bh
    ex = bh.NativeExecutor()
    yield ex


@pytest.fixture
def gpu_rt(gpu_executor):
    import bohrium_b200 as bh
    return bh.Runtime(gpu_executor)


@pytest.fixture
def oracle_rt():
    import bohrium_b200 as bh
    from oracle.ve_openmp import OracleExecutor
    return bh.Runtime(OracleExecutor(threads=min(8, os.cpu_count() or 1)))
