import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from checkers import REFERENCE_TREE  # noqa: E402  (KESSLER_REFERENCE, else the default tree)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: longer CPU checks")


@pytest.fixture(scope="session")
def ks():
    """The engine package (loads libkessler_b200.so; fails loudly if missing)."""
    mod = importlib.import_module("kessler-syndrom-simulation_b200")
    mod.load_library()
    return mod


@pytest.fixture(scope="session")
def oracle():
    import checkers
    if not os.path.exists(checkers.ORACLE_SO):
        checkers.build(ref=False)
    return checkers.Oracle()


@pytest.fixture(scope="session")
def reference():
    import checkers
    if not checkers.reference_available():
        if os.path.isdir(os.path.join(REFERENCE_TREE, "src")):
            checkers.build(ref=True)
        else:
            pytest.skip("reference build (oracle/_ref) not available")
    return checkers.Reference()


@pytest.fixture(scope="session")
def engine(ks):
    eng = ks.Engine(0)
    yield eng
    eng.close()


def golden_path(name):
    return os.path.join(ROOT, "tests", "golden", name)
