"""Failure detection on the device without a fault: an armed context makes one TMA line copy of
the rows transform wait for bytes that never come, so that bounded wait expires (a short poll
budget), the kernel reports it through the context's error word, drains its own copies with the
full budget and ends.  The host sees HH_ERR_DEVICE; the context and the request loop keep
working, and the next calls give the oracle's results again."""
import numpy as np
import pytest
from conftest import rel_err

import hackathon_b200 as hh

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_expired_wait_is_reported_and_the_context_recovers(ctx, oracle):
    n, rows = 255, 64
    rng = np.random.default_rng(5)
    x = rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))
    src = torch.from_numpy(x).cuda()
    dst = torch.zeros_like(src)
    ctx.synchronize()
    ctx.inject_wait_expiry()
    ctx.dst1_rows(n, rows, src, dst)
    with pytest.raises(hh.HHError, match="HH_ERR_DEVICE"):
        ctx.synchronize()
    ctx.synchronize()  # reported once, then cleared
    ctx.dst1_rows(n, rows, src, dst)  # the injection was taken by one launch only
    ctx.synchronize()
    torch.cuda.synchronize()
    assert rel_err(dst.cpu().numpy(), oracle.dst1_rows(x)) < 1e-13


def test_expired_wait_fails_its_request_in_the_loop(ctx):
    # the loop's plans take the tuning cache's settings; without an entry they keep the length's
    # default rows kernel, which is the one the injection is armed in
    hh.tune_cache_clear()
    n, nrhs = 255, 2
    rng = np.random.default_rng(6)
    f = rng.standard_normal((nrhs, n, n)) + 1j * rng.standard_normal((nrhs, n, n))
    plan = hh.Plan.helmholtz(ctx, 2, n, 6, 12.0)
    plan.apply_tuning()  # the settings the request loop's plan of this shape takes
    solo = plan.solve_source_host(f)
    plan.close()
    srv = hh.Server(0, hbm_budget=2 << 30, streams=2)
    fp = torch.from_numpy(f).pin_memory()
    outs = [torch.empty_like(fp).pin_memory() for _ in range(4)]
    srv.wait(srv.submit(2, n, 6, 12.0, nrhs, fp, outs[0]))
    srv.inject_wait_expiry()
    bad = srv.submit(2, n, 6, 12.0, nrhs, fp, outs[1])
    with pytest.raises(hh.HHError, match="HH_ERR_DEVICE"):
        srv.wait(bad)  # a failed request, not a hang
    for i in (2, 3):
        srv.wait(srv.submit(2, n, 6, 12.0, nrhs, fp, outs[i]))
    srv.close()
    for i in (0, 2, 3):
        assert np.array_equal(outs[i].numpy(), solo)
