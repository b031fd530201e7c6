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
assembled right-hand sides) on the whole field.  Each direction is one all_to_all_single for the
whole batch over the process group (NCCL between GPUs), laid out so that the forward exchange
lands in the pencil and the pencil goes back as it is: the pencil interleaves the right-hand
sides row by row ([z][b][line], solved by hh_solve_lines_strided), and the only copies are the
cut of the transformed slab into the ranks' lines before the exchange and the reassembly of the
planes after it, one kernel each (hh_lines_pack).  The
steps of one rank are separate methods, so that a test can run several ranks in one process with
the exchange done by hand.
"""

from __future__ import annotations

import contextlib

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
        """pencil: [n, B, lines] (z rows of the rank's lines, right-hand sides interleaved row by
        row), solved in place."""
        nb, cnt = pencil.shape[1], pencil.shape[2]
        self.plan.solve_lines_strided(pencil, pencil, nb, self.fused, nb * cnt, cnt)

    def pack(self, slab, send, world: int):
        """send <- slab [B, planes, n, n] cut into the world ranks' lines, rank s's part
        [planes][B][lines_s], the parts in rank order (hh_lines_pack)."""
        self.ctx.lines_pack(slab, send, slab.shape[0], slab.shape[1], self.n * self.n, world)

    def unpack(self, back, slab, world: int):
        self.ctx.lines_pack(back, slab, slab.shape[0], slab.shape[1], self.n * self.n, world, unpack=True)

    def close(self):
        self.plan.close()
        self.ctx.close()


class SlabPencil3D:
    """Rank `rank` of `world` in a slab/pencil solve of n^3 fields (see the module docstring).

    Exchange buffers, one all_to_all_single each way for the whole batch of B right-hand sides:

    * send: the transformed slab cut into the ranks' lines, rank s's part [planes][B][lines_s],
      the parts in rank order;
    * pencil [n, B, lines]: the z rows of this rank's lines, right-hand sides interleaved row by
      row, so that what rank s sends is rows [z0_s, z1_s), contiguous: the forward exchange lands
      in place and the pencil goes back as it is;
    * back: rank s's pencil rows of this rank's planes, [planes][B][lines_s], in rank order.
    """

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

    def slab_counts(self, batch: int) -> list:
        """Elements per peer in the slab-side buffers (send, back)."""
        z0, z1 = self.planes
        return [(z1 - z0) * batch * (b - a) for a, b in self.qs]

    def pencil_counts(self, batch: int) -> list:
        """Elements per peer in the pencil."""
        q0, q1 = self.lines
        return [(b - a) * batch * (q1 - q0) for a, b in self.zs]

    def send_piece(self, send, s: int, batch: int):
        """Rank s's part of a send (or back) buffer, [planes][B][lines_s]."""
        counts = self.slab_counts(batch)
        off = sum(counts[:s])
        q0, q1 = self.qs[s]
        return send[off:off + counts[s]].view(self.planes[1] - self.planes[0], batch, q1 - q0)

    back_piece = send_piece

    def pencil_piece(self, pencil, s: int):
        """Rows of rank s's planes in the pencil, [planes_s][B][lines]."""
        z0, z1 = self.zs[s]
        return pencil[z0:z1]

    # -- the three steps of one rank
    def to_pencils(self, f, slab):
        """slab <- the transform of the source planes f, both [B, planes, n, n]; returns the send
        buffer."""
        import torch
        with self._on_steps_stream():
            self.steps.forward(f, slab)
            send = torch.empty(sum(self.slab_counts(slab.shape[0])), dtype=slab.dtype, device=slab.device)
            self.steps.pack(slab, send, self.world)
            return send

    def new_pencil(self, batch: int, like):
        import torch
        q0, q1 = self.lines
        with self._on_steps_stream():
            return torch.empty((self.n, batch, q1 - q0), dtype=like.dtype, device=like.device)

    def new_back(self, batch: int, like):
        import torch
        with self._on_steps_stream():
            return torch.empty(sum(self.slab_counts(batch)), dtype=like.dtype, device=like.device)

    def solve_pencil(self, pencil):
        """The z line solves of the pencil [n, B, lines], in place."""
        with self._on_steps_stream():
            self.steps.lines(pencil)

    def to_slab(self, back, out):
        """The back buffer into out [B, planes, n, n], which is then transformed back in place."""
        with self._on_steps_stream():
            self.steps.unpack(back, out, self.world)
            self.steps.inverse(out)

    # -- the whole solve over a process group
    def solve(self, f, u, group=None):
        """u <- the solution's planes of this rank's slab from the source planes f, both
        [B, planes, n, n] complex128 tensors; every rank of the group calls it together."""
        import torch
        import torch.distributed as dist
        nb = f.shape[0]
        sl = [2 * c for c in self.slab_counts(nb)]
        pc = [2 * c for c in self.pencil_counts(nb)]
        with self._on_steps_stream():
            send = self.to_pencils(f, u)
            pencil = self.new_pencil(nb, u)
            dist.all_to_all_single(torch.view_as_real(pencil).reshape(-1), torch.view_as_real(send).reshape(-1),
                                   pc, sl, group=group)
            self.solve_pencil(pencil)
            back = self.new_back(nb, u)
            dist.all_to_all_single(torch.view_as_real(back).reshape(-1), torch.view_as_real(pencil).reshape(-1),
                                   sl, pc, group=group)
            self.to_slab(back, u)


def solve_in_process(ranks: list, fs: list, us: list):
    """All ranks of a decomposition in one process, the exchanges done by hand: rank r's slab of
    the sources fs[r] -> us[r].  One GPU (or the CPU) runs the ranks' steps one after another; no
    step of one rank waits for another's."""
    world, nb = len(ranks), fs[0].shape[0]
    sends = [rk.to_pencils(f, u) for rk, f, u in zip(ranks, fs, us)]
    pencils = [rk.new_pencil(nb, u) for rk, u in zip(ranks, us)]
    for r, rk in enumerate(ranks):      # receiver
        for s in range(world):          # sender
            with rk._on_steps_stream():
                rk.pencil_piece(pencils[r], s).copy_(ranks[s].send_piece(sends[s], r, nb))
    for rk, p in zip(ranks, pencils):
        rk.solve_pencil(p)
    backs = [rk.new_back(nb, u) for rk, u in zip(ranks, us)]
    for r, rk in enumerate(ranks):
        for s in range(world):
            with rk._on_steps_stream():
                rk.back_piece(backs[r], s, nb).copy_(ranks[s].pencil_piece(pencils[s], r))
    for rk, bk, u in zip(ranks, backs, us):
        rk.to_slab(bk, u)
