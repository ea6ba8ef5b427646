"""Shared test set-up: markers, build of the oracle (the checker) and of the
in-tree CUDA library, scene fixtures."""
import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import pyoracle
    pyoracle.build(with_ref=True)
    return pyoracle


@pytest.fixture(scope="session")
def upf_lib():
    from unifiedparticleframeworkcuda_b200 import build
    build.build()
    import unifiedparticleframeworkcuda_b200 as upf
    upf.lib()
    return upf
