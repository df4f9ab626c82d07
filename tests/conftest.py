import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libteide_ref.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def gpu():
    """td.h binding of the product library (libteide_b200.so) on the GPU."""
    import teide_b200
    td = teide_b200.load()
    if td.lib.td_gpu_device_count() <= 0:
        pytest.fail("no CUDA device visible: the GPU tests need one")
    return td


@pytest.fixture(scope="session")
def td():
    """td.h binding of the product library for host-side calls (no GPU needed)."""
    import teide_b200
    return teide_b200.load()


@pytest.fixture(scope="session")
def ref():
    """td.h binding of Teide itself, compiled from its sources (checker)."""
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref/libteide_ref.so not built")
    from teide_b200.td import Td
    return Td(REF_LIB)
