"""GPU parity at the benchmark configurations themselves (the same generators, seeds, sizes and
batches the benchmark uses), against the oracle, which is bit-exact with the reference's C path
(tests/test_oracle.py), and against the manufactured exact solution where the source has one:

* 3D N=255, order 6, k=30, a batch of 4 right-hand sides of 16 sine modes (p, q, r <= 64);
* 2D N=1023, orders {4, 6} x k {10, 50, 200}, a batch of 64 right-hand sides of 32 sine modes
  (p, q <= 200) plus CN(0, 1e-3) noise per point;
* 2D N=2047, order 6, k in {10, 100, 400} (the k = 400 lines are not diagonally dominant), a
  batch of 16 right-hand sides of 8 sine modes (p, q <= 20).

Each batch is solved in one call; the oracle checks two of its right-hand sides (the first and
the last), which is where a batching or chunking error would show.  Tolerance: 1e-12 relative
(max|u - u_ref| / max|u_ref|), with the extended-precision fallback of
conftest.assert_parity_2d for near-resonant 2D lines."""
import numpy as np
import pytest
from conftest import assert_parity_2d, rel_err

import hackathon_b200 as hh
from hackathon_b200 import workload as W

pytestmark = pytest.mark.gpu

TOL = 1e-12


def test_config_3d_n255_o6_k30_batch4(ctx, oracle):
    n, order, k, batch = 255, 6, 30.0, 4
    modes = [W.sine_modes(2000 + b, 16, 64, dim=3) for b in range(batch)]
    f_ext = [W.source_3d(n, m) for m in modes]
    f = np.stack([x[1:-1, 1:-1, 1:-1] for x in f_ext])
    plan = hh.Plan.helmholtz(ctx, 3, n, order, k)
    plan.tune(batch)
    u = plan.solve_source_host(f)
    plan.close()
    for b in (0, batch - 1):
        ref = oracle.pipeline_3d(n, order, k, f_ext[b])
        assert rel_err(u[b], ref["sol"]) < TOL, b
        exact = W.exact_3d(n, modes[b], k)
        e_gpu, e_ref = rel_err(u[b], exact), rel_err(ref["sol"], exact)
        # the same discrete solution, so the same error against the exact one: by the triangle
        # inequality the two differ by at most max|u - u_ref| / max|exact| ~ TOL
        assert abs(e_gpu - e_ref) <= 1.5 * TOL, (e_gpu, e_ref)
        assert e_gpu < 1e-4  # 6th order at h = 1/256 with modes up to 64 (the oracle: 1.2e-5)


@pytest.mark.parametrize("order", [4, 6])
def test_config_2d_n1023_batch64(ctx, oracle, order):
    n, batch = 1023, 64
    f_ext = [W.source_2d(n, W.sine_modes(1000 + b, 32, 200), noise_seed=1000 + b + 0x1000000, noise_var=1e-3,
                         fast=True) for b in range(batch)]
    f = np.stack([x[1:-1, 1:-1] for x in f_ext])
    for k in (10.0, 50.0, 200.0):
        plan = hh.Plan.helmholtz(ctx, 2, n, order, k)
        plan.tune(batch)
        u = plan.solve_source_host(f)
        plan.close()
        for b in (0, batch - 1):
            ref = oracle.pipeline_2d(n, order, k, f_ext[b])
            assert_parity_2d(oracle, u[b], ref, TOL)


def test_config_2d_n2047_o6_batch16(ctx, oracle):
    n, order, batch = 2047, 6, 16
    modes = [W.sine_modes(3000 + b, 8, 20) for b in range(batch)]
    f_ext = [W.source_2d(n, m, fast=True) for m in modes]
    f = np.stack([x[1:-1, 1:-1] for x in f_ext])
    for k in (10.0, 100.0, 400.0):
        plan = hh.Plan.helmholtz(ctx, 2, n, order, k)
        plan.tune(batch)
        u = plan.solve_source_host(f)
        plan.close()
        for b in (0, batch - 1):
            ref = oracle.pipeline_2d(n, order, k, f_ext[b])
            assert_parity_2d(oracle, u[b], ref, TOL)
            exact = W.exact_2d(n, modes[b], k)
            e_gpu, e_ref = rel_err(u[b], exact), rel_err(ref["sol"], exact)
            assert abs(e_gpu - e_ref) <= 1.5 * TOL, (k, e_gpu, e_ref)
            # 6th order at h = 1/2048 with modes up to 20: the discretisation error is at the
            # rounding level (the oracle: 2e-12 at k = 10, 3e-13 at k = 400 on the first one)
            assert e_gpu < 1e-10
