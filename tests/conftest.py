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


def assert_parity_2d(oracle, u, ref: dict, tol: float = 1e-12):
    """Parity of a GPU solution with the reference's FP64 result.

    Passes when max|u - u_ref| / max|u_ref| <= tol.  Otherwise the case is ill-conditioned
    enough that the reference's own rounding error exceeds tol: the solution is then compared
    with the exact solution of the same discrete system (extended-precision solve) and must be
    at least as accurate as the reference, within a factor 1.5 (+1e-14)."""
    e = rel_err(u, ref["sol"])
    if e <= tol:
        return e
    truth = oracle.solver_2d_ld(ref["coef"], ref["rhs"])
    e_ref, e_gpu = rel_err(ref["sol"], truth), rel_err(u, truth)
    assert e_gpu <= 1.5 * e_ref + 1e-14, f"rel err vs reference {e:.3e}; vs exact: gpu {e_gpu:.3e}, reference {e_ref:.3e}"
    return e


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
