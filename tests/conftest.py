import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200)')


@pytest.fixture(scope='session')
def oracle():
    from oracle import COracle
    return COracle()


@pytest.fixture(scope='session')
def reference():
    """Grappolo's own functions (oracle/_ref); skipped where they were not built."""
    from oracle.lvoracle import HERE
    if not os.path.exists(os.path.join(HERE, '_ref', 'libgrappolo_ref.so')):
        pytest.skip('reference library not built (oracle/_ref)')
    from oracle import Reference
    return Reference()
