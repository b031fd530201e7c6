"""The request loop (include/hh.h hh_server_*): a mixed stream of 2D/3D requests, merged into
batches (requests of one shape at any k share a batch) and spread over streams, gives every
request exactly the result of a solo solve."""
import numpy as np
import pytest

import hackathon_b200 as hh

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _requests(seed, count):
    rng = np.random.default_rng(seed)
    sizes = [(2, 63), (2, 127), (2, 255), (3, 15), (3, 31)]
    out = []
    for i in range(count):
        dim, n = sizes[rng.integers(len(sizes))]
        order = int(rng.choice([2, 4, 6]))
        k = float(rng.choice([5.0, 20.0, 37.5]))  # few distinct k so that requests share plans
        nrhs = int(rng.integers(1, 5))
        shape = (nrhs,) + (n,) * dim
        f = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        out.append((dim, n, order, k, nrhs, f))
    return out


def _solo(ctx, dim, n, order, k, f):
    """The request alone: a plan of its own with the kernel settings the request loop's plans take
    (the tuning cache's entry for the shape, if the process has one)."""
    plan = hh.Plan.helmholtz(ctx, dim, n, order, k)
    plan.apply_tuning()
    u = plan.solve_source_host(f)
    plan.close()
    return u


def test_mixed_stream_matches_solo_host_buffers(ctx):
    # the mixed stream, then a burst of requests of one plan (queued behind each other, so the
    # loop has same-plan requests waiting to merge); buffers are pinned before submission so that
    # submitting is fast next to solving
    rng = np.random.default_rng(11)
    burst = [(2, 63, 4, 5.0, 2, rng.standard_normal((2, 63, 63)) + 1j * rng.standard_normal((2, 63, 63)))
             for _ in range(8)]
    reqs = _requests(1, 40) + burst
    bufs = []
    for dim, n, order, k, nrhs, f in reqs:
        fp = torch.from_numpy(f).pin_memory()
        bufs.append((fp, torch.empty_like(fp).pin_memory()))
    srv = hh.Server(0, hbm_budget=8 << 30, streams=3)
    ids = [srv.submit(dim, n, order, k, nrhs, fp, up) for (dim, n, order, k, nrhs, f), (fp, up) in zip(reqs, bufs)]
    infos = [srv.wait(i) for i in ids]
    stats = srv.stats()
    srv.close()
    assert stats["completed"] == len(reqs)
    merged = 0
    for (dim, n, order, k, nrhs, f), (fp, up), info in zip(reqs, bufs, infos):
        assert info["t_submit"] <= info["t_start"] <= info["t_done"]
        merged += info["batch_rhs"] > nrhs
        assert np.array_equal(up.numpy(), _solo(ctx, dim, n, order, k, f))  # alone == in the mix
    assert merged > 0  # continuous batching happened


def test_device_buffers_and_direct_path(ctx):
    reqs = _requests(2, 12)
    srv = hh.Server(0, hbm_budget=8 << 30, streams=2)
    bufs, ids = [], []
    for dim, n, order, k, nrhs, f in reqs:
        fd = torch.from_numpy(f).cuda()
        ud = torch.empty_like(fd)
        bufs.append((fd, ud))
        ids.append(srv.submit(dim, n, order, k, nrhs, fd, ud, on_device=True))
    for i in ids:
        srv.wait(i)
    srv.close()
    for (dim, n, order, k, nrhs, f), (fd, ud) in zip(reqs, bufs):
        assert np.array_equal(ud.cpu().numpy(), _solo(ctx, dim, n, order, k, f))


def test_budget_admission_and_rejection(ctx):
    n, nrhs = 255, 4
    rng = np.random.default_rng(3)
    f = rng.standard_normal((nrhs, n, n)) + 1j * rng.standard_normal((nrhs, n, n))
    one = nrhs * n * n * 16
    # room for about one request at a time: every request still completes, one after another
    srv = hh.Server(0, hbm_budget=int(2.5 * one) + (8 << 20), streams=4)
    fp = torch.from_numpy(f).pin_memory()
    outs = [torch.empty_like(fp).pin_memory() for _ in range(6)]
    ids = [srv.submit(2, n, 6, 10.0 + i, nrhs, fp, outs[i]) for i in range(6)]  # one shape, six plans
    infos = [srv.wait(i) for i in ids]
    for i, u in enumerate(outs):
        assert np.array_equal(u.numpy(), _solo(ctx, 2, n, 6, 10.0 + i, f))
    # batches over several k are cut to what the budget admits: staging plus the plans they create
    plan_bytes = 2 * n * n * 16 + n * 4096 + (1 << 20)
    budget = int(2.5 * one) + (8 << 20)
    assert all(b["batch_rhs"] // nrhs * (one + plan_bytes) <= budget for b in infos)
    # a request that can never fit is refused, and the server keeps working afterwards
    big = torch.empty((64, n, n), dtype=torch.complex128).pin_memory()
    bad = srv.submit(2, n, 6, 99.0, 64, big, big)
    with pytest.raises(hh.HHError, match="HH_ERR_NOMEM"):
        srv.wait(bad)
    ok = srv.submit(2, n, 6, 10.0, nrhs, fp, outs[0])
    srv.wait(ok)
    srv.close()
    assert np.array_equal(outs[0].numpy(), _solo(ctx, 2, n, 6, 10.0, f))


def test_injected_failure_fails_only_its_batch(ctx):
    """A batch whose error word is set (host-side injection, as if one of its kernels had seen a
    bounded wait expire) fails with HH_ERR_DEVICE; the batches after it, on the same stream and
    on the others, succeed with the solo result: every stream's word is cleared per batch."""
    n, nrhs = 63, 2
    rng = np.random.default_rng(9)
    f = rng.standard_normal((nrhs, n, n)) + 1j * rng.standard_normal((nrhs, n, n))
    solo = _solo(ctx, 2, n, 4, 7.0, f)
    srv = hh.Server(0, hbm_budget=2 << 30, streams=2)
    fp = torch.from_numpy(f).pin_memory()
    outs = [torch.empty_like(fp).pin_memory() for _ in range(5)]
    first = srv.submit(2, n, 4, 7.0, nrhs, fp, outs[0])
    srv.wait(first)  # the plan exists; the next request runs alone
    srv.inject_error(1)
    bad = srv.submit(2, n, 4, 7.0, nrhs, fp, outs[1])
    with pytest.raises(hh.HHError, match="HH_ERR_DEVICE"):
        srv.wait(bad)
    for i in range(2, 5):  # both streams, round robin: each succeeds
        srv.wait(srv.submit(2, n, 4, 7.0, nrhs, fp, outs[i]))
    srv.close()
    for i in (0, 2, 3, 4):
        assert np.array_equal(outs[i].numpy(), solo)
