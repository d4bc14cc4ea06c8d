import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through the C ABI")
    config.addinivalue_line("markers", "fullsize: a benchmark configuration at its full size (minutes; also gpu)")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (built on first use)."""
    from oracle import pyoracle
    pyoracle.orc()
    return pyoracle


@pytest.fixture(scope="session")
def reflib(oracle):
    """The reference's own physics headers compiled by oracle/Makefile (`make ref`)."""
    lib = oracle.ref()
    if lib is None:
        pytest.skip("oracle/_ref not built (needs the reference checkout at build time)")
    return lib
