"""Test configuration: the ``gpu`` marker and session-wide builds.

Tests marked ``gpu`` need a B200 (sm_100); everything else runs on the CPU.
The session fixture builds the CUDA library (nvcc cross-compiles without a
GPU) and the C++ oracle before any test imports them.
"""
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    from solvix_b200 import build as b
    b.build()
    from oracle import oracle
    oracle.build()
    yield


@pytest.fixture(scope="session")
def ctx():
    """One device context for the whole GPU session."""
    from solvix_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(autouse=True)
def _oracle_sort_mode():
    """Every test starts with the oracle in the reference's row order."""
    from oracle import oracle
    oracle.set_sort_mode(0)
    yield
    oracle.set_sort_mode(0)
