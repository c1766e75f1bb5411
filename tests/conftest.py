"""Shared pytest configuration.

Marker `gpu`: needs a CUDA device (run on the B200 box with `-m gpu`).
Everything else runs on a CPU-only machine.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def engine_lib():
    """The engine library (built in-tree if missing; nvcc cross-compiles without a GPU)."""
    from psdm_b200 import build
    build.build()
    from psdm_b200 import _lib
    return _lib.lib()


@pytest.fixture(scope="session")
def engine(engine_lib):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from psdm_b200.rtm import Engine
    e = Engine(0)
    yield e
    e.close()
