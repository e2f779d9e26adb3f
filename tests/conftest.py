import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
ORACLE_DIR = os.path.join(ROOT, "oracle")
if ORACLE_DIR not in sys.path:
    sys.path.insert(0, ORACLE_DIR)

REF_LIB = os.path.join(ORACLE_DIR, "_ref", "libhmsbeagle.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: full-size workloads")


def _pkg():
    return importlib.import_module("beagle-lib_b200")


@pytest.fixture(scope="session")
def pkg():
    return _pkg()


@pytest.fixture(scope="session")
def syn(pkg):
    return pkg.synthetic


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o


@pytest.fixture(scope="session")
def reflib(pkg):
    """The reference BEAGLE CPU library compiled by oracle/Makefile, if present."""
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref not built (make -C oracle)")
    return pkg.binding.BeagleLib(REF_LIB, "beagle")


@pytest.fixture(scope="session")
def b200(pkg):
    """libbeagle_b200.so; on a GPU run a missing library fails loudly."""
    return pkg.load()
