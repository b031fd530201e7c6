"""The slab/pencil 3D decomposition (hackathon_b200/slab_pencil.py) on the CPU.  Its exchanges
run as gloo ranks (or by hand in one process); each rank's compute steps are the oracle's
transform along x and y and the reference's Thomas recurrence along z
(3D_Program/solver_functions/solver.c:483-496) with its LU() factors, on the rank's own lines.
The ranks' slabs, put together, must give the reference's one-process solve (ora_solver_3d)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp
from conftest import rel_err

from hackathon_b200 import slab_pencil as SP
from hackathon_b200 import workload as W

TOL = 1e-12


class OracleSteps:
    """A rank's compute steps on the CPU (test infrastructure): the oracle's DST along x and y, and
    the reference's Thomas solve on lines [q0, q1) with the factors of its LU()."""

    def __init__(self, n, L, U, Up, q0, q1):
        from oracle import Oracle
        self.o, self.n = Oracle(), n
        cut = lambda a: np.ascontiguousarray(a.reshape(n * n, n)[q0:q1].T)  # [z, line]
        self.L, self.U, self.Up = cut(L), cut(U), cut(Up)

    def _x(self, a):
        return self.o.dst1_rows(a)

    def _y(self, a):
        return np.swapaxes(self.o.dst1_rows(np.ascontiguousarray(np.swapaxes(a, -1, -2))), -1, -2)

    def forward(self, src, slab):
        slab.copy_(torch.from_numpy(np.ascontiguousarray(self._y(self._x(src.numpy())))))

    def inverse(self, slab):
        slab.copy_(torch.from_numpy(np.ascontiguousarray(self._x(self._y(slab.numpy())))))

    def pack(self, slab, send, world):
        nb, planes = slab.shape[:2]
        flat, off = slab.reshape(nb, planes, -1), 0
        for q0, q1 in SP.split(flat.shape[2], world):
            cnt = planes * nb * (q1 - q0)
            send[off:off + cnt] = flat[:, :, q0:q1].permute(1, 0, 2).reshape(cnt)
            off += cnt

    def unpack(self, back, slab, world):
        nb, planes = slab.shape[:2]
        flat, off = slab.view(nb, planes, -1), 0
        for q0, q1 in SP.split(flat.shape[2], world):
            cnt = planes * nb * (q1 - q0)
            flat[:, :, q0:q1] = back[off:off + cnt].reshape(planes, nb, q1 - q0).permute(1, 0, 2)
            off += cnt

    def lines(self, pencil):
        p = pencil.numpy()  # [z][b][line]
        nz = p.shape[0]
        for b in range(p.shape[1]):
            r = p[:, b]
            y = np.empty_like(r)
            y[0] = r[0]
            for l in range(1, nz):
                y[l] = r[l] - self.L[l] * y[l - 1]
            x = np.empty_like(r)
            x[nz - 1] = y[nz - 1] * self.U[nz - 1]
            for l in range(nz - 2, -1, -1):
                x[l] = (y[l] - self.Up[l] * x[l + 1]) * self.U[l]
            p[:, b] = x


def _problem(n, order, k, batch):
    from oracle import Oracle
    o = Oracle()
    rhs, sol = [], []
    for b in range(batch):
        ref = o.pipeline_3d(n, order, k, W.source_3d(n, W.sine_modes(5 * n + b, 8, min(n, 12), dim=3)))
        rhs.append(ref["rhs"])
        sol.append(ref["sol"])
    L, U, Up = o.lu_3d(n, n, n, ref["coef"])
    return np.stack(rhs), np.stack(sol), (L, U, Up)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, n, rhs, fac, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        z0, z1 = SP.split(n, world)[rank]
        q0, q1 = SP.split(n * n, world)[rank]
        rk = SP.SlabPencil3D(n, rank, world, OracleSteps(n, *fac, q0, q1))
        f = torch.from_numpy(np.ascontiguousarray(rhs[:, z0:z1]))
        u = torch.empty_like(f)
        rk.solve(f, u)
        out[rank] = u.numpy()
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_split_is_balanced_and_contiguous():
    for total, parts in [(255, 4), (255 * 255, 8), (7, 7), (10, 3)]:
        s = SP.split(total, parts)
        assert s[0][0] == 0 and s[-1][1] == total
        assert all(a[1] == b[0] for a, b in zip(s, s[1:]))
        sizes = [b - a for a, b in s]
        assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    with pytest.raises(ValueError):
        SP.split(3, 4)


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_ranks_in_one_process_match_reference(world):
    """Uneven splits of planes and lines (n = 15 over 2, 3 and 5 ranks), exchanges by hand."""
    n, batch = 15, 2
    rhs, sol, fac = _problem(n, 6, 10.0, batch)
    ranks, fs, us = [], [], []
    for r in range(world):
        z0, z1 = SP.split(n, world)[r]
        q0, q1 = SP.split(n * n, world)[r]
        ranks.append(SP.SlabPencil3D(n, r, world, OracleSteps(n, *fac, q0, q1)))
        fs.append(torch.from_numpy(np.ascontiguousarray(rhs[:, z0:z1])))
        us.append(torch.empty_like(fs[-1]))
    SP.solve_in_process(ranks, fs, us)
    u = np.concatenate([x.numpy() for x in us], axis=1)
    assert rel_err(u, sol) < TOL


def test_two_gloo_ranks_match_reference():
    """The exchange as all_to_all_single between two processes (gloo)."""
    n, batch, world = 15, 2, 2
    rhs, sol, fac = _problem(n, 4, 30.0, batch)
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, n, rhs, fac, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=240)
            assert p.exitcode == 0
        res = dict(out)
    u = np.concatenate([res[r] for r in range(world)], axis=1)
    assert rel_err(u, sol) < TOL
