import glob
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through librbffd_sm100.so")
    config.addinivalue_line("markers", "slow: longer CPU test")


def has_gpu():
    """Decided from the device nodes, not from the library: on a GPU machine a
    missing or broken librbffd_sm100.so must fail the gpu tests, not skip them."""
    return os.path.exists("/dev/nvidiactl") or bool(glob.glob("/dev/nvidia[0-9]*"))


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def ctx():
    import rbffd_gpu_b200 as R
    c = R.Context(0)
    yield c
    c.close()
