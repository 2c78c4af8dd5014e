"""Test configuration: the `gpu` marker and on-demand builds of the CUDA
library (randomfield_b200/librf_b200.so) and of the CPU oracle
(oracle/librfo.so)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU; runs the CUDA path through the C-ABI")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from oracle import oracle

    oracle.lib()  # builds librfo.so when missing or stale
    from randomfield_b200 import build

    build.build()
    yield
