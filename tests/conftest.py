import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_ROOT = "/root/reference"
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cb05():
    from camp_b200.mechanism import Mechanism

    return Mechanism.load(os.path.join(GOLDEN, "cb05cl_ae5.mech.json"))


@pytest.fixture(scope="session")
def cb05_ref():
    return dict(np.load(os.path.join(GOLDEN, "cb05cl_ae5_ref.npz")))


@pytest.fixture(scope="session")
def lib():
    from camp_b200 import build, _lib

    build.build()
    return _lib.load()
