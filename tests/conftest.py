import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a) and libps2cuda.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(GOLDEN / name)

    return load


@pytest.fixture(scope="session")
def cuda_lib():
    """The product library; GPU tests fail (not skip) when it is missing."""
    from pystamps_b200 import build
    from pystamps_b200 import _lib

    build.build()
    return _lib.lib()
