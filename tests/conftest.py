import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on a B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.bindings import Checker
    return Checker("oracle")


@pytest.fixture(scope="session")
def ref():
    from oracle.bindings import Checker, reference_available
    if not reference_available():
        pytest.skip("reference host build unavailable (no reference tree on this machine)")
    return Checker("ref")


@pytest.fixture(scope="session")
def config0():
    from lsystemeditor_b200.scene import config0_scene
    return config0_scene()


@pytest.fixture(scope="session")
def tracer():
    """GPU renderer through the C ABI; fails loudly when CUDA or the library is missing."""
    from lsystemeditor_b200.pathtracer import PathTracer
    t = PathTracer(0)
    yield t
    t.close()
