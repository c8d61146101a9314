"""Shared test setup.

Markers: ``gpu`` -- needs a CUDA device (run with ``-m gpu``); everything else
runs on a CPU-only machine.  The oracle (oracle/, test infrastructure) is the
checker for every GPU result.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, build_oracle
    build_oracle()
    return Oracle()


@pytest.fixture(scope="session")
def cuda_lib():
    """The product library, built if missing; requires a GPU to be used."""
    import torch
    from cagr_b200 import build as B
    if not os.path.exists(B.LIB_PATH):
        B.build()
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cagr_b200 import _lib
    return _lib.lib()
