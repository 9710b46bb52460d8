import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU checks")


@pytest.fixture(scope="session")
def oracle():
    from tests.oracle_libs import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from tests.oracle_libs import Reference, reference_available
    if not reference_available():
        pytest.skip("reference library not built (oracle/_ref/libmpcdref.so needs the reference sources)")
    return Reference()
