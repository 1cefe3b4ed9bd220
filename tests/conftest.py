import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def arena_mesh():
    from rocketgpu_b200 import arena
    return arena.generate()


@pytest.fixture(scope="session")
def oracle_available():
    from tests import oracle_ref
    if not oracle_ref.available():
        pytest.skip("oracle not built (make -C oracle)")
    return True
