import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_small(name):
    return dict(np.load(os.path.join(GOLDEN, f"small_{name}.npz")))


def load_sym(name):
    return dict(np.load(os.path.join(GOLDEN, f"sym_{name}.npz")))


SMALL_CASES = ["grid2d_20", "grid3d_8", "stencil27_4", "grid2d_100"]


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
