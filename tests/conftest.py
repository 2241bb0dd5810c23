import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    import oracle

    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        oracle.build(with_reference=None)
    yield


def needs_reference(T=1):
    import oracle

    return pytest.mark.skipif(not oracle.ref_available(T), reason="reference CPU library (oracle/_ref) not built")
