import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


@pytest.fixture(scope="session")
def harm_lib():
    from harm_cool_b200 import build, library
    build.build()
    return library()


@pytest.fixture(scope="session")
def oracle_built():
    from oracle import build_oracle
    return build_oracle.build()


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
