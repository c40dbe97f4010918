"""Shared fixtures: the product library (libcaelix_b200.so through its ctypes binding), the CPU
oracle (oracle/liboracle.so, the checker) and a CUDA device. Tests marked `gpu` need a B200."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "caelix-renderer_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)
if os.path.join(REPO, "tests") not in sys.path:
    sys.path.insert(0, os.path.join(REPO, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import oracle_lib

    return oracle_lib.load()


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    import caelix_b200

    dev = caelix_b200.Device(0)
    yield dev
    dev.close()
