"""The slab/pencil 3D decomposition on the GPU (hackathon_b200/slab_pencil.py): every rank's steps
run on cuda:0 one after another, or as the single rank of an NCCL group.  Each plane and line goes
through the arithmetic of the one-process solve, so the ranks' slabs put together are bitwise the
one-process hh_solve_source / hh_solve of the whole field."""
import datetime
import os
import socket

import numpy as np
import pytest

import hackathon_b200 as hh
from hackathon_b200 import slab_pencil as SP

pytestmark = pytest.mark.gpu


def _fields(n, batch, seed):
    import torch
    g = torch.Generator().manual_seed(seed)
    shape = (batch, n, n, n)
    return torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                         torch.randn(shape, generator=g, dtype=torch.float64)).cuda()


def _ranks(n, order, k, world, fused, variant):
    import torch
    stream, out = torch.cuda.Stream(0), []
    for r in range(world):
        q0, q1 = SP.split(n * n, world)[r]
        out.append(SP.SlabPencil3D(n, r, world, SP.DeviceSteps(0, n, order, k, q0, q1, fused, variant, stream)))
    return out


@pytest.mark.parametrize("n,order,k,batch", [(31, 6, 10.0, 3), (63, 4, 30.0, 2), (47, 2, 20.0, 2),
                                             (127, 6, 30.0, 2), (255, 6, 30.0, 1)])
@pytest.mark.parametrize("world", [2, 3, 8])
@pytest.mark.parametrize("fused", [True, False])
def test_ranks_in_one_process_bitwise_one_process_solve(ctx, n, order, k, batch, world, fused):
    import torch
    f = _fields(n, batch, 31 * n + world)
    plan = hh.Plan.helmholtz(ctx, 3, n, order, k)
    ref = torch.full_like(f, float("nan"))
    torch.cuda.synchronize()
    (plan.solve_source if fused else plan.solve)(f, ref, batch)
    ctx.synchronize()
    ranks = _ranks(n, order, k, world, fused, plan.variant)
    fs, us = [], []
    for rk in ranks:
        z0, z1 = rk.planes
        fs.append(f[:, z0:z1].contiguous())
        us.append(torch.full_like(fs[-1], float("nan")))
    SP.solve_in_process(ranks, fs, us)
    torch.cuda.synchronize()
    u = torch.cat(us, dim=1)
    assert torch.isfinite(u).all()
    assert torch.equal(u, ref)
    for rk in ranks:
        rk.steps.close()
    plan.close()


@pytest.mark.parametrize("batch,planes,nlines,world", [(3, 5, 961, 3), (1, 32, 65025, 8), (2, 7, 100, 7)])
def test_lines_pack_layout_and_round_trip(ctx, batch, planes, nlines, world):
    """hh_lines_pack against torch slicing of the same layout, and unpack(pack(x)) == x."""
    import torch
    g = torch.Generator().manual_seed(nlines + world)
    x = torch.complex(torch.randn((batch, planes, nlines), generator=g, dtype=torch.float64),
                      torch.randn((batch, planes, nlines), generator=g, dtype=torch.float64)).cuda()
    send = torch.full((batch * planes * nlines,), float("nan"), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    ctx.lines_pack(x, send, batch, planes, nlines, world)
    ctx.synchronize()
    off = 0
    for q0, q1 in SP.split(nlines, world):  # rank s's part [planes][batch][lines_s]
        cnt = planes * batch * (q1 - q0)
        assert torch.equal(send[off:off + cnt].reshape(planes, batch, q1 - q0), x[:, :, q0:q1].permute(1, 0, 2))
        off += cnt
    y = torch.full_like(x, float("nan"))
    torch.cuda.synchronize()
    ctx.lines_pack(send, y, batch, planes, nlines, world, unpack=True)
    ctx.synchronize()
    assert torch.equal(y, x)
    with pytest.raises(hh.HHError):
        ctx.lines_pack(x, x, batch, planes, nlines, world)
    with pytest.raises(hh.HHError):
        ctx.lines_pack(x, send, batch, planes, nlines, nlines + 1)


def test_strided_line_solve_interleaved_equals_contiguous(ctx):
    """hh_solve_lines_strided on fields interleaved row by row ([z][b][line]) gives the bits of
    hh_solve_lines on the same fields one after another ([b][z][line]); overlapping layouts are
    refused."""
    import torch
    n, batch = 63, 3
    g = torch.Generator().manual_seed(63)
    f = torch.complex(torch.randn((batch, n, n * n), generator=g, dtype=torch.float64),
                      torch.randn((batch, n, n * n), generator=g, dtype=torch.float64)).cuda()
    p = hh.Plan.helmholtz(ctx, 3, n, 6, 20.0)
    a = f.clone()
    b = f.permute(1, 0, 2).contiguous()
    torch.cuda.synchronize()
    p.solve_lines(a, a, batch)
    p.solve_lines_strided(b, b, batch, True, batch * n * n, n * n)
    ctx.synchronize()
    assert torch.isfinite(a).all()
    assert torch.equal(b.permute(1, 0, 2), a)
    with pytest.raises(hh.HHError):
        p.solve_lines_strided(b, b, batch, True, n * n, n * n)  # fields would overlap
    p.close()


def test_line_range_plan_only_solves_lines(ctx):
    import torch
    p = hh.Plan.helmholtz_lines(ctx, 31, 6, 10.0, 100, 500)
    assert p.field == 400 * 31
    x = torch.zeros(p.field, dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    for call in (lambda: p.solve_source(x, x, 1), lambda: p.solve(x, x, 1), lambda: p.tune(1)):
        with pytest.raises(hh.HHError):
            call()
    with pytest.raises(hh.HHError):
        hh.Plan.helmholtz_lines(ctx, 31, 6, 10.0, 500, 100)
    with pytest.raises(hh.HHError):
        hh.Plan.helmholtz_lines(ctx, 31, 6, 10.0, 0, 31 * 31 + 1)
    p.solve_lines(x, x, 1)
    ctx.synchronize()
    p.close()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_nccl_group_of_one(ctx):
    """SlabPencil3D.solve through NCCL's all_to_all_single (a group of one rank on this GPU)."""
    import torch
    import torch.distributed as dist
    n, order, k, batch = 63, 6, 20.0, 2
    f = _fields(n, batch, 7)
    plan = hh.Plan.helmholtz(ctx, 3, n, order, k)
    ref = torch.empty_like(f)
    torch.cuda.synchronize()
    plan.solve_source(f, ref, batch)
    ctx.synchronize()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        rk = SP.SlabPencil3D(n, 0, 1, SP.DeviceSteps(0, n, order, k, 0, n * n, True, plan.variant))
        u = torch.full_like(f, float("nan"))
        torch.cuda.synchronize()
        rk.solve(f, u)
        torch.cuda.synchronize()
        assert torch.equal(u, ref)
        rk.steps.close()
    finally:
        dist.destroy_process_group()
    plan.close()
