import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a library")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (C restatement), built on demand."""
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    import pyoracle

    return pyoracle


@pytest.fixture(scope="session")
def ks():
    """The product package with its CUDA library loaded (no fallback)."""
    import solver_cpp_b200 as ks

    ks.lib()
    return ks


@pytest.fixture(scope="session")
def ctx(ks):
    c = ks.Context(0)
    yield c
    c.close()
