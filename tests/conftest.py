import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def orc():
    import pyoracle
    return pyoracle


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "reference_goldens.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def beams():
    return dict(np.load(os.path.join(GOLDEN, "beams.npz")))


@pytest.fixture(scope="session")
def built_lib():
    from pofd_affine_b200 import build
    build.build()
    return build.LIB


@pytest.fixture(scope="session")
def gpu_ctx(built_lib):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    from pofd_affine_b200 import Context
    return Context(0)


@pytest.fixture(scope="session")
def host_ctx(built_lib):
    from pofd_affine_b200 import Context
    return Context(-1)
