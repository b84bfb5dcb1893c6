"""Test configuration.

Markers: ``gpu`` tests need a B200 (sm_100) and call the CUDA library through
the C ABI; everything else runs on CPU. Oracle libraries (oracle/_build,
oracle/_ref) are test infrastructure and are only loaded here.
"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "nabla-ai_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU; calls the CUDA library")


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle.Restatement()


@pytest.fixture(scope="session")
def ref():
    import oracle
    return oracle.Reference()


@pytest.fixture(scope="session")
def ctx():
    from nabla_b200 import solver
    return solver.default_context()
