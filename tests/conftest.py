"""Shared test setup: the `gpu` marker, the in-tree library and oracle builds.

`-m "not gpu"` runs on a machine without a GPU (oracle against the golden
vectors, host logic, the C ABI's exports). `-m gpu` runs the parity tests
through the C ABI on a B200.
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def libso():
    from clsparse_b200 import _lib
    if not _lib.LIB_PATH.exists():
        from clsparse_b200 import build
        build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def cuda(libso):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


@pytest.fixture()
def ctrl(cuda):
    from clsparse_b200 import api
    c = api.Control()
    yield c
    c.release()
