"""Shared fixtures.  Tests marked `gpu` need a B200; everything else runs on
the CPU (oracle vs golden fixtures, host logic, C-ABI exports)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device (B200)")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(GOLDEN, "golden_small.npz")))


@pytest.fixture(scope="session")
def bank():
    from broccoli_b200 import filters as F
    return F.load_filter_dir(os.path.join(GOLDEN, "filters"))


@pytest.fixture(scope="session")
def lin_filters(bank):
    return bank["linear"]


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from broccoli_b200.api import Context
    c = Context(0)
    yield c
    torch.cuda.synchronize()
    c.close()


def rel_err(a, b):
    """max |a - b| / max |b| (norm-wise relative error)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))
