"""hh_solve_source_host_noalloc: the host-buffer solve for callers that must not allocate device
memory while they run; its staging is the library's fixed device array.  Collected last (file
name), so it also runs after every other GPU test."""
import numpy as np
import pytest

import hackathon_b200 as hh
from hackathon_b200 import workload as W

pytestmark = pytest.mark.gpu


def _f(n, seed):
    return W.source_2d(n, W.sine_modes(seed, 8, 20), noise_seed=seed + 1, noise_var=1e-3)[1:-1, 1:-1]


@pytest.mark.parametrize("n,order,k,batch", [(1023, 6, 50.0, 2), (511, 4, 100.0, 8), (255, 6, 10.0, 5)])
def test_noalloc_equals_allocating_solve_twice(ctx, n, order, k, batch):
    plan = hh.Plan.helmholtz(ctx, 2, n, order, k)
    for call in range(2):  # two calls in a row: nothing carries over between them
        f = np.stack([_f(n, 100 * call + b) for b in range(batch)])
        want = plan.solve_source_host(f)
        got = plan.solve_source_host_noalloc(f)
        assert np.array_equal(got, want)
    plan.close()


def test_noalloc_3d_and_rejection(ctx):
    n = 63
    plan = hh.Plan.helmholtz(ctx, 3, n, 6, 30.0)
    f = W.source_3d(n, W.sine_modes(9, 8, 16, dim=3))[1:-1, 1:-1, 1:-1]
    assert np.array_equal(plan.solve_source_host_noalloc(f), plan.solve_source_host(f))
    plan.close()
    big = hh.Plan.helmholtz(ctx, 2, 1023, 6, 50.0)
    with pytest.raises(hh.HHError, match="HH_ERR_UNSUPPORTED"):
        big.solve_source_host_noalloc(np.zeros((3, 1023, 1023), dtype=np.complex128))  # over 2^21 values
    big.close()


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


def test_noalloc_first_call_on_a_fresh_context():
    """The allocation-free call as the very first solve of a new context (every table it needs
    was made when the plan was created), then again, against the allocating entry point.  The
    device's free memory is the same before and after each of the two calls: neither call
    allocates, the first included."""
    pytest.importorskip("torch")
    _free_bytes()  # the runtime's own first-use set-up happens here, outside the checks
    ctx = hh.Context(0)
    n = 1023
    plan = hh.Plan.helmholtz(ctx, 2, n, 4, 30.0)
    f1, f2 = _f(n, 7), _f(n, 8)
    before = _free_bytes()
    got1 = plan.solve_source_host_noalloc(f1)
    after1 = _free_bytes()
    got2 = plan.solve_source_host_noalloc(f2)
    after2 = _free_bytes()
    assert before == after1 == after2, (before, after1, after2)
    assert np.array_equal(got1, plan.solve_source_host(f1))
    assert np.array_equal(got2, plan.solve_source_host(f2))
    plan.close()
    ctx.close()
