"""Shared pytest configuration.

Markers: `gpu` -- needs a CUDA device (run on a B200 with `-m gpu`); all
other tests run on CPU.  The oracle under oracle/ is the checker only.
"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "k-litho_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    torch.cuda.init()
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def ref_built():
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference build oracle/_ref not present (needs the reference checkout)")
    return O
