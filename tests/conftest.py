import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle.Oracle()


@pytest.fixture(scope="session")
def reference_lib():
    import oracle
    oracle.build()
    if not oracle.reference_available("strict"):
        pytest.skip("compiled reference (oracle/_ref) not available on this host")
    return oracle.Reference("strict")
