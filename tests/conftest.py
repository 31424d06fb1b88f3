"""Test configuration: the `gpu` marker, repository imports and shared
fixtures.  Tests without the marker run on CPU only (oracle, host logic and
the C-ABI library's symbol table)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C-ABI")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def gx():
    """The engine package with its library built and a default context."""
    import gacelle_b200
    from gacelle_b200 import build
    build.build()
    gacelle_b200.lib()
    return gacelle_b200


@pytest.fixture(scope="session")
def ctx(gx):
    return gx.Context.default(0)
