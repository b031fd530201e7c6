"""A 3D solve split over ranks: z-slabs for the transforms, (i, j)-line pencils for the line solves.

The reference solves a 3D field in one process (3D_Program/solver_functions/solver.c:263-413): a
2D DST of every z plane, Thomas along z on every (i, j) line, the inverse 2D DST.  Split over R
ranks, one per GPU (the decomposition of the paper the reference accompanies, Algorithm 2):

* rank r holds planes [z0_r, z1_r) of every right-hand side (its slab) for the transforms, and
  lines [q0_r, q1_r) of the n^2 lines, q = i + j n, for the line solves (its pencil);
1. the x and y transforms of its planes (hh_dst1_rows, then hh_dst1_cols: the plan's forward
   transform);
2. all-to-all: rank s receives the lines of its pencil from every plane of every slab;
3. the z line solves of its pencil (hh_solve_lines on a line-range plan,
   hh_plan3d_create_helmholtz_lines);
4. all-to-all back: rank s receives the planes of its slab from every pencil;
5. the inverse transforms (columns, then rows, as the plan's inverse).

Every plane and every line goes through exactly the arithmetic of the one-process solve, so with
the same line-solve variant the result is bitwise that of hh_solve_source (or of hh_solve, for
assembled right-hand sides) on the whole field.  Each exchange is one all_to_all_single over the
process group (NCCL between GPUs).  The steps of one rank are separate methods, so that a test can
run several ranks in one process with the exchange done by hand.
"""

from __future__ import annotations

import contextlib

import numpy as np

from . import Context, Plan


def split(total: int, parts: int) -> list[tuple[int, int]]:
    """[begin, end) of each of `parts` contiguous, balanced ranges of range(total)."""
    if parts < 1 or total < parts:
        raise ValueError(f"cannot split {total} into {parts} non-empty ranges")
    base, extra = divmod(total, parts)
    out, a = [], 0
    for r in range(parts):
        b = a + base + (1 if r < extra else 0)
        out.append((a, b))
        a = b
    return out


class DeviceSteps:
    """One rank's compute steps on its GPU: the library's transforms over the slab and a line-range
    plan over the pencil.  They run on `stream` (a torch.cuda.Stream; a new one if None), which
    SlabPencil3D also gives the exchange's copies and collectives, ordered behind the caller's
    stream on entry and ahead of it on return.  Ranks run in one process share one stream."""

    def __init__(self, device: int, n: int, order: int, k: complex, q0: int, q1: int, fused: bool = True,
                 variant: int | None = None, stream=None):
        import torch
        self.stream = stream if stream is not None else torch.cuda.Stream(device)
        self.ctx = Context(device, stream=self.stream.cuda_stream)
        self.n, self.fused = n, fused
        self.plan = Plan.helmholtz_lines(self.ctx, n, order, k, q0, q1)
        if variant is not None:
            self.plan.variant = variant

    def forward(self, src, slab):
        """src, slab: [B, planes, n, n] complex128 on the device; slab <- src transformed along x,
        then y (src may be slab)."""
        n, planes = self.n, slab.shape[0] * slab.shape[1]
        self.ctx.dst1_rows(n, planes * n, src, slab)
        self.ctx.dst1_cols(n, n, planes, slab, n, n * n, slab)

    def inverse(self, slab):
        n, planes = self.n, slab.shape[0] * slab.shape[1]
        self.ctx.dst1_cols(n, n, planes, slab, n, n * n, slab)
        self.ctx.dst1_rows(n, planes * n, slab, slab)

    def lines(self, pencil):
        """pencil: [B, n, lines] (z rows of the rank's lines), solved in place."""
        self.plan.solve_lines(pencil, pencil, pencil.shape[0], self.fused)

    def close(self):
        self.plan.close()
        self.ctx.close()


class SlabPencil3D:
    """Rank `rank` of `world` in a slab/pencil solve of n^3 fields (see the module docstring)."""

    def __init__(self, n: int, rank: int, world: int, steps):
        self.n, self.rank, self.world, self.steps = n, rank, world, steps
        self.zs = split(n, world)
        self.qs = split(n * n, world)

    @contextlib.contextmanager
    def _on_steps_stream(self):
        """Run the enclosed torch work on the steps' stream (device steps), ordered behind the
        caller's stream and ahead of it afterwards."""
        s = getattr(self.steps, "stream", None)
        if s is None:
            yield
            return
        import torch
        caller = torch.cuda.current_stream(s.device)
        s.wait_stream(caller)
        with torch.cuda.stream(s):
            yield
        caller.wait_stream(s)

    @property
    def planes(self) -> tuple[int, int]:
        return self.zs[self.rank]

    @property
    def lines(self) -> tuple[int, int]:
        return self.qs[self.rank]

    # -- the three steps of one rank; chunks are lists indexed by the peer rank
    def to_pencils(self, f, slab) -> list:
        """slab <- the transform of the source planes f, both [B, planes, n, n]; chunk s holds rank
        s's lines of it, [B, planes, lines_s]."""
        with self._on_steps_stream():
            self.steps.forward(f, slab)
            flat = slab.reshape(slab.shape[0], slab.shape[1], self.n * self.n)
            return [flat[:, :, q0:q1].contiguous() for q0, q1 in self.qs]

    def pencil_shapes(self, batch: int) -> list:
        q0, q1 = self.lines
        return [(batch, z1 - z0, q1 - q0) for z0, z1 in self.zs]

    def solve_pencil(self, recv: list) -> list:
        """recv[s]: [B, planes_s, lines] from rank s.  Solves the pencil [B, n, lines]; chunk s
        holds rank s's planes of it."""
        import torch
        with self._on_steps_stream():
            pencil = torch.cat(recv, dim=1).contiguous()
            self.steps.lines(pencil)
            return [pencil[:, z0:z1, :].contiguous() for z0, z1 in self.zs]

    def slab_shapes(self, batch: int) -> list:
        z0, z1 = self.planes
        return [(batch, z1 - z0, q1 - q0) for q0, q1 in self.qs]

    def to_slab(self, recv: list, out):
        """recv[s]: [B, planes, lines_s] from rank s, written into out [B, planes, n, n], which is
        then transformed back in place."""
        with self._on_steps_stream():
            flat = out.view(out.shape[0], out.shape[1], self.n * self.n)
            for (q0, q1), part in zip(self.qs, recv):
                flat[:, :, q0:q1] = part
            self.steps.inverse(out)

    # -- the whole solve over a process group
    def solve(self, f, u, group=None):
        """u <- the solution's planes of this rank's slab from the source planes f, both
        [B, planes, n, n] complex128 tensors; every rank of the group calls it together."""
        b = f.shape[0]
        with self._on_steps_stream():
            recv = exchange(self.to_pencils(f, u), self.pencil_shapes(b), group)
            recv = exchange(self.solve_pencil(recv), self.slab_shapes(b), group)
            self.to_slab(recv, u)


def exchange(chunks: list, recv_shapes: list, group=None) -> list:
    """One all_to_all_single: chunk s goes to rank s; returns the chunks received, shaped as
    recv_shapes (complex128)."""
    import torch
    import torch.distributed as dist
    send = torch.cat([torch.view_as_real(c).reshape(-1) for c in chunks])
    sizes_in = [2 * c.numel() for c in chunks]
    sizes_out = [2 * int(np.prod(s)) for s in recv_shapes]
    recv = torch.empty(sum(sizes_out), dtype=torch.float64, device=send.device)
    dist.all_to_all_single(recv, send, sizes_out, sizes_in, group=group)
    return [torch.view_as_complex(p.view(*s, 2)) for p, s in zip(torch.split(recv, sizes_out), recv_shapes)]


def solve_in_process(ranks: list, fs: list, us: list):
    """All ranks of a decomposition in one process, the exchanges done by hand: rank r's slab of
    the sources fs[r] -> us[r].  One GPU (or the CPU) runs the ranks' steps one after another; no
    step of one rank waits for another's."""
    world = len(ranks)
    sends = [rk.to_pencils(f, u) for rk, f, u in zip(ranks, fs, us)]
    backs = [rk.solve_pencil([sends[s][r] for s in range(world)]) for r, rk in enumerate(ranks)]
    for r, (rk, u) in enumerate(zip(ranks, us)):
        rk.to_slab([backs[s][r] for s in range(world)], u)
