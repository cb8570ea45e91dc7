import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


@pytest.fixture(scope="session")
def fg():
    """The CUDA backend (fails loudly when the extension is missing)."""
    import ferray_b200
    ferray_b200.default_context()
    return ferray_b200


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.lib()
    return o
