import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device (B200)")


@pytest.fixture(scope="session")
def product_lib():
    """The built libmpzmm_b200.so (built in place if missing)."""
    from rforest_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    return _lib.lib()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    if not os.path.exists(O.LIB_ORACLE):
        O.build(with_reference=False)
    return O


@pytest.fixture(scope="session")
def gpu(product_lib):
    """Set up the device; a GPU test fails (never skips to a fallback) when the
    CUDA path is unavailable."""
    from rforest_b200 import api
    api.setup(0)
    return product_lib
