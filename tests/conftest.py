"""Test configuration: the `gpu` marker, in-tree builds and shared fixtures.

CPU tests (`-m "not gpu"`) cover the oracle against the reference's golden
vectors and known answers, the host logic, and the C ABI library's exports.
GPU tests (`-m gpu`) are the parity tests proper: they call the CUDA path
through the C ABI and compare it with the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    from mcls_b200 import build
    from oracle import oracle

    build.build()
    oracle.build()
    yield


@pytest.fixture(scope="session")
def ctx():
    from mcls_b200 import capi

    c = capi.Context(0)
    yield c
    c.close()
