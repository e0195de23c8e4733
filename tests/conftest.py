import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the product kernels")


@pytest.fixture(scope="session")
def nxg_lib():
    from nanoxgen_b200 import build
    build.build_library()
    from nanoxgen_b200 import _abi
    return _abi.lib()


@pytest.fixture(scope="session")
def oracle():
    from oracle.checker import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.checker import Reference, reference_available
    if not reference_available():
        pytest.skip("reference checkout absent and oracle/_ref not prebuilt")
    return Reference()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test ran without a CUDA device")
    return torch.device("cuda:0")
