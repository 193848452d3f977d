import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on the CPU")


def golden(name):
    with open(os.path.join(HERE, "golden", name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle():
    from checkers import Checker
    return Checker("oracle")


@pytest.fixture(scope="session")
def reference():
    from checkers import REF_SO, REFERENCE_TREE, Checker
    if not os.path.exists(REF_SO) and not os.path.isdir(REFERENCE_TREE):
        pytest.skip("reference build not available")
    return Checker("ref")


@pytest.fixture(scope="session")
def lib():
    import pevsl_b200
    from pevsl_b200 import build as b
    if not os.path.exists(pevsl_b200.LIB_PATH):
        b.build()
    return pevsl_b200.load()


@pytest.fixture(scope="session")
def gpu():
    """The CUDA path; GPU tests fail (not skip) when the library is missing."""
    import pevsl_b200
    lib = pevsl_b200.load()
    buf = pevsl_b200.info()
    assert "sm_100a" in buf
    return lib
