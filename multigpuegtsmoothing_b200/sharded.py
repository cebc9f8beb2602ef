"""Row-partitioned Taubin smoothing over several ranks (one GPU per rank).

The reference smooths on several GPUs by giving each card a contiguous range
of the sorted points and exchanging, every half-step, the positions of the
neighbours that other cards own (EGT_CUDA.cu:293-474 builds the halo lists,
:559-607 sends and receives them between the lambda and mu steps, :636-646
gathers every card's range at the end).  This module does the same over
torch.distributed:

* ShardPlan partitions the rows of the filtered neighbourhood CSR into
  contiguous ranges, one per rank, and precomputes once what each rank needs
  from, and sends to, every other rank.  The CSR is known to every rank (the
  reference replicates the cloud on every card too), so no communication is
  needed to build the plan.
* ShardedTaubin keeps a rank's own rows followed by its halo in one float4
  array.  Each half-step receives the halo positions (grouped point-to-point
  sends and receives: one NCCL group over NVLink with the nccl backend), then
  runs the half-step over the rank's rows (egt_taubin_halfstep: the same
  per-row arithmetic, in list order, as the single-GPU loop), and finally
  all-gathers the ranges.

A row's new position depends only on its own and its neighbours' positions
before the half-step, in list order, so the partitioned result equals the
single-GPU one bit for bit.  There is no multicast: every remote position lands
in the rank's own memory before it is read.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple

import numpy as np


class ShardPlan:
    """Partition of CSR rows [0, n) into `world` contiguous ranges and the halo
    lists of rank `rank`.

    Attributes (numpy int arrays unless noted):
      lo, hi           the rank's rows [lo, hi)
      off, col         the rank's local CSR: rows 0..hi-lo-1, columns indexing
                       the local position array (own rows first, then the halo)
      halo             global ids of the halo, ascending (grouped by owner)
      recv             per peer: (start, count) of its block in the halo
      send             per peer: local row indices the peer needs from this rank
    """

    def __init__(self, csr_off: np.ndarray, csr_col: np.ndarray, world: int, rank: int,
                 bounds: Optional[np.ndarray] = None):
        off = np.asarray(csr_off, dtype=np.int64)
        col = np.asarray(csr_col, dtype=np.int64)
        n = off.shape[0] - 1
        if not (0 <= rank < world):
            raise ValueError("rank out of range")
        if bounds is None:
            bounds = np.array([n * r // world for r in range(world + 1)], dtype=np.int64)
        bounds = np.asarray(bounds, dtype=np.int64)
        if bounds.shape[0] != world + 1 or bounds[0] != 0 or bounds[-1] != n or np.any(np.diff(bounds) < 0):
            raise ValueError("bounds must rise from 0 to n, one range per rank")
        self.world, self.rank, self.n = world, rank, n
        self.bounds = bounds
        self.lo, self.hi = int(bounds[rank]), int(bounds[rank + 1])
        self.halo, local_col = self._local(off, col, self.lo, self.hi)
        self.off = (off[self.lo:self.hi + 1] - off[self.lo]).astype(np.int32)
        self.col = local_col.astype(np.int32)
        owner = np.searchsorted(bounds, self.halo, side="right") - 1
        self.recv: List[Tuple[int, int]] = []
        for p in range(world):
            idx = np.nonzero(owner == p)[0]
            self.recv.append((int(idx[0]), int(idx.size)) if idx.size else (0, 0))
        # what every peer needs from this rank: its halo entries inside [lo, hi)
        self.send: List[np.ndarray] = []
        for p in range(world):
            if p == rank:
                self.send.append(np.zeros(0, np.int64))
                continue
            plo, phi = int(bounds[p]), int(bounds[p + 1])
            cols = col[off[plo]:off[phi]]
            mine = np.unique(cols[(cols >= self.lo) & (cols < self.hi)])
            self.send.append(mine - self.lo)

    @staticmethod
    def _local(off, col, lo, hi):
        cols = col[off[lo]:off[hi]]
        outside = (cols < lo) | (cols >= hi)
        halo = np.unique(cols[outside])
        local = np.empty_like(cols)
        local[~outside] = cols[~outside] - lo
        local[outside] = (hi - lo) + np.searchsorted(halo, cols[outside])
        return halo, local

    @property
    def rows(self) -> int:
        return self.hi - self.lo


def cuda_halfstep(pos_in, pos_out, off, col, rows: int, scale: float):
    """The GPU half-step over a rank's rows (egt_taubin_halfstep) on torch
    CUDA tensors, on torch's current stream."""
    import ctypes as C

    import torch
    from . import capi
    st = torch.cuda.current_stream().cuda_stream
    capi._check(capi.lib().egt_taubin_halfstep(C.c_void_p(pos_in.data_ptr()), C.c_void_p(pos_out.data_ptr()),
                                               C.c_void_p(off.data_ptr()), C.c_void_p(col.data_ptr()), int(rows),
                                               float(scale), int(pos_in.device.index or 0),
                                               C.c_void_p(st) if st else None))


class ShardedTaubin:
    """Taubin lambda/mu smoothing of the rank's rows with halo exchange.

    positions: (n, 4) float32 tensor of every point (x, y, z, w) -- the
    replicated starting positions; plan: this rank's ShardPlan; halfstep: the
    per-rank half-step (cuda_halfstep by default; any callable with its
    signature); group: the torch.distributed process group (None = default).
    """

    def __init__(self, positions, plan: ShardPlan, halfstep: Optional[Callable] = None, group=None):
        import torch
        self.plan = plan
        self.group = group
        self.halfstep = halfstep or cuda_halfstep
        dev = positions.device
        self.dev = dev
        m = plan.rows + plan.halo.shape[0]
        self.local = torch.empty((m, 4), dtype=torch.float32, device=dev)
        self.local[:plan.rows] = positions[plan.lo:plan.hi]
        self.local[plan.rows:] = positions[torch.as_tensor(plan.halo, device=dev, dtype=torch.long)]
        self.out = torch.empty((plan.rows, 4), dtype=torch.float32, device=dev)
        self.off = torch.as_tensor(plan.off, device=dev)
        self.col = torch.as_tensor(plan.col, device=dev)
        self.send_idx = [torch.as_tensor(s, device=dev, dtype=torch.long) for s in plan.send]
        self.send_buf = [torch.empty((s.shape[0], 4), dtype=torch.float32, device=dev) for s in plan.send]

    def exchange(self):
        """Receives the halo positions of this half-step from their owners
        (grouped sends and receives, every rank in the same order)."""
        import torch.distributed as dist
        if self.plan.world == 1:
            return
        ops = []
        for p in range(self.plan.world):
            if p == self.plan.rank:
                continue
            start, cnt = self.plan.recv[p]
            if self.send_idx[p].numel():
                self.send_buf[p].copy_(self.local[self.send_idx[p]])
                ops.append(dist.P2POp(dist.isend, self.send_buf[p], p, group=self.group))
            if cnt:
                ops.append(dist.P2POp(dist.irecv, self.local[self.plan.rows + start:self.plan.rows + start + cnt],
                                      p, group=self.group))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()

    def run(self, iters: int, lam: float = 0.63, mu: float = -0.64):
        for _ in range(iters):
            for scale in (lam, mu):
                self.exchange()
                self.halfstep(self.local, self.out, self.off, self.col, self.plan.rows, scale)
                self.local[:self.plan.rows].copy_(self.out)

    def gather(self):
        """Every rank's rows, all-gathered into (n, 4) positions on every rank
        (the reference's final copy between cards, EGT_CUDA.cu:636-646)."""
        import torch
        import torch.distributed as dist
        if self.plan.world == 1:
            return self.local[:self.plan.rows].clone()
        sizes = np.diff(self.plan.bounds)
        width = int(sizes.max())
        mine = torch.zeros((width, 4), dtype=torch.float32, device=self.dev)
        mine[:self.plan.rows] = self.local[:self.plan.rows]
        parts = [torch.empty_like(mine) for _ in range(self.plan.world)]
        dist.all_gather(parts, mine, group=self.group)
        return torch.cat([parts[r][:int(sizes[r])] for r in range(self.plan.world)])
