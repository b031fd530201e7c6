"""The multi-GPU form is replicas: every rank solves its own seeded batch and the job's time is
the slowest rank's.  The host-side logic of that (bench.py: aggregate_over_ranks and the
per-rank inputs) runs here as two gloo ranks on the CPU."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        def reduce_max(x: float) -> float:
            t = torch.tensor([x], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())

        ms_max, value = bench.aggregate_over_ranks(10.0 + 5.0 * rank, 64, 30, world, reduce_max)
        # the first right-hand side of this rank's batch: seeded by the rank, so ranks differ
        f0 = bench.sources(1, index=1 + rank)[0]
        digest = torch.tensor([float(np.abs(f0).sum())], dtype=torch.float64)
        gathered = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, digest)
        out[rank] = (ms_max, value, [float(g.item()) for g in gathered])
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=240)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        ms_max, value, digests = res[r]
        assert ms_max == 15.0  # the slower rank bounds the job
        assert value == pytest.approx(world * 64 * 30 / 0.015)
        assert digests[0] != digests[1]  # each rank solves its own inputs
    assert res[0][2] == res[1][2]


def test_single_rank_needs_no_collective():
    import bench
    ms_max, value = bench.aggregate_over_ranks(12.5, 64, 10, 1, lambda x: pytest.fail("no collective at N=1"))
    assert ms_max == 12.5 and value == pytest.approx(64 * 10 / 0.0125)
