import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA kernels through the C-ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle("strict")


@pytest.fixture(scope="session")
def renderer():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mandelbulber2_b200.render import Renderer

    r = Renderer(0)
    yield r
    r.close()
