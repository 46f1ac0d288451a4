import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = "geos-chem-gpu-hybrid_b200"
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libraries")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module(PKG)


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.load("fullchem")
    return oracle


@pytest.fixture(scope="session")
def mech():
    from mechanism import codegen
    return codegen.load("fullchem")
