"""Shared pytest setup.

GPU tests are marked ``gpu`` and run on a B200; everything else runs on CPU.
The package directory and the oracle directory are put on sys.path here.
"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "blender-lucid-renderer_b200")
ORACLE = os.path.join(REPO, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle_ctypes
    return oracle_ctypes.load()


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("scenes"))
