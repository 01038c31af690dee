import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / 'golden'
sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200) and the built libsawsim_b200.so')


@pytest.fixture(scope='session')
def built_lib():
    """Build (or reuse) the in-tree shared library."""
    from sawsim_b200 import build
    return build.build()
