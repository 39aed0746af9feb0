"""Shared pytest setup.

Marker ``gpu``: the test needs a B200 and the in-tree CUDA library; the CPU
suite runs ``-m "not gpu"``.  The CPU oracle (oracle/) is importable from
every test as ``import oracle``.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU and the built CUDA library")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def cuda():
    """The product package with its library loaded (GPU tests only)."""
    import n_body_sim_pro_b200 as nb

    nb.library()
    return nb


@pytest.fixture()
def ctx(cuda):
    c = cuda.CudaContext()
    yield c
    c.close()
