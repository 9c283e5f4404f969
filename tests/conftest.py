import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a)')
    config.addinivalue_line('markers', 'slow: long-running CPU replay of a recorded tape')


@pytest.fixture(scope='session')
def oracle_lib():
    from tests import helpers
    return helpers.oracle()


@pytest.fixture(scope='session')
def ref_lib():
    from tests import helpers
    r = helpers.reference()
    if r is None:
        pytest.skip('oracle/_ref (the reference kernels translated to C++) is not built here')
    return r


@pytest.fixture(scope='session')
def kernels_meta():
    from tests import helpers
    return helpers.kernels_meta()
