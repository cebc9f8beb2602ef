"""The partitioned smoothing's per-rank GPU step (egt_taubin_halfstep) on one GPU.

Two row ranges of one cloud are smoothed as two ranks would smooth them, in
one process: each keeps its rows and halo in its own float4 array, the halo is
refreshed from the other range before every half-step (what the ranks' grouped
sends and receives do), and the CUDA half-step runs on each range.  The ranges
put together must equal egt_taubin on the whole cloud bit for bit; one range
covering everything must too.  (No two kernels here wait on each other: the
ranks are emulated one after the other.)
"""
import numpy as np
import pytest

from multigpuegtsmoothing_b200 import datagen

pytestmark = pytest.mark.gpu


def _setup(capi, iters):
    xyz = datagen.superquadrics(200_000, seed=83)
    g = capi.GridStructure(xyz)
    g.GRIDCUDAKNNSELF_COMPACT(40)
    e = capi.EGT_CUDA(g)
    e.Filter(0.65)
    start = g.sorted_positions()
    off, col = g.csr()
    e.Taubin(iters)
    want = g.sorted_positions()
    g.close()
    pos4 = np.zeros((start.shape[1], 4), np.float32)
    pos4[:, :3] = start.T
    return pos4, off, col, want


@pytest.mark.parametrize("world", [1, 2])
def test_halfstep_ranges_equal_whole_cloud(capi, world):
    import torch
    from multigpuegtsmoothing_b200.sharded import ShardPlan, ShardedTaubin
    iters = 10
    pos4, off, col, want = _setup(capi, iters)
    dev = torch.device("cuda", 0)
    full = torch.from_numpy(pos4).to(dev)
    parts = [ShardedTaubin(full, ShardPlan(off, col, world, r)) for r in range(world)]

    def refresh_halo():
        owned = torch.empty_like(full)
        for p in parts:
            owned[p.plan.lo:p.plan.hi] = p.local[:p.plan.rows]
        for p in parts:
            if p.plan.halo.size:
                p.local[p.plan.rows:] = owned[torch.as_tensor(p.plan.halo, device=dev, dtype=torch.long)]

    for _ in range(iters):
        for scale in (0.63, -0.64):
            refresh_halo()
            for p in parts:
                p.halfstep(p.local, p.out, p.off, p.col, p.plan.rows, scale)
                p.local[:p.plan.rows].copy_(p.out)
    torch.cuda.synchronize()
    got = torch.cat([p.local[:p.plan.rows] for p in parts]).cpu().numpy()
    assert np.array_equal(got[:, :3].T, want)
