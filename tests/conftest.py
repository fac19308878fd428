import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ref_mhd():
    from oracle import ref
    if not ref.available(True):
        pytest.fail("oracle library missing: run `make -C oracle` (needs the reference sources)")
    return ref.Reference(True)


@pytest.fixture(scope="session")
def ref_hydro():
    from oracle import ref
    if not ref.available(False):
        pytest.fail("oracle library missing: run `make -C oracle` (needs the reference sources)")
    return ref.Reference(False)
