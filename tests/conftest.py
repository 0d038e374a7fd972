import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA integrator")


@pytest.fixture(scope="session")
def port():
    from oracle import oracle as O
    if not os.path.exists(O.PORT_PATH):
        O.build()
    return O.port()


@pytest.fixture(scope="session")
def ref():
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference library oracle/_ref not built (reference sources absent)")
    return O.ref()
