import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "anisotropic-ml_b200")
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long CPU test")


def load_case(name):
    z = np.load(os.path.join(GOLDEN, f"case_{name}.npz"))
    return {k: z[k] for k in z.files}


def load_model(name):
    z = np.load(os.path.join(GOLDEN, f"model_{name}.npz"))
    n = len(z.files) // 2
    return [(z[f"W{k}"], z[f"b{k}"]) for k in range(n)]


def case_model(case):
    return load_model(bytes(case["model"]).decode()[len("model_"):])


def case_shape(case):
    from oracle.shapes import SHAPES
    return SHAPES[bytes(case["shape"]).decode()]


@pytest.fixture(scope="session")
def cuda_available():
    import torch
    return torch.cuda.is_available()
