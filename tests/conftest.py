import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200)')


@pytest.fixture(scope='session')
def oracle_bins():
    from oracle import build as ob
    return ob.build()


@pytest.fixture(scope='session')
def gpu_lib():
    from coseis_b200 import build as b
    b.build()
    from coseis_b200 import _lib
    return _lib.load()
