import os
import sys
import pathlib

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def lib():
    from adcirc_b200 import build, _lib
    build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build()
    return oracle
