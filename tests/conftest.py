import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, 'oracle'))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200); runs the CUDA kernels')


@pytest.fixture(scope='session')
def oracle_mod():
    import oracle as O
    O.load()
    return O


@pytest.fixture(scope='session')
def cuda_lib():
    """The CUDA library, built if needed; GPU tests fail (not skip) without it."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail('GPU test run without a CUDA device')
    from clvisc_b200 import _lib, build
    build.build()
    return _lib.load()
