import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the libfoggy_b200 kernels")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "inline_goldens.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def native():
    """The CUDA library; a GPU test fails (never skips) when it cannot be loaded."""
    from itofoggysim_b200 import build, _native
    build.build()
    return _native.load()
