import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


def rel_err(a, b) -> float:
    """max |a - b| / max |b| (the parity measure used throughout)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name))


def have_ref() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref2d.so"))


@pytest.fixture(scope="session")
def ctx():
    import hackathon_b200 as hh
    c = hh.Context(0)
    yield c
    c.close()
