"""Row-partitioned Taubin smoothing with halo exchange, on CPU gloo ranks.

multigpuegtsmoothing_b200.sharded partitions the filtered neighbourhood CSR
over ranks, exchanges halo positions before every half-step and all-gathers
the ranges at the end, as the reference does across cards (EGT_CUDA.cu:293-474,
559-646).  Here 2 and 3 gloo ranks on 127.0.0.1 run it with the oracle's FP32
half-step in place of the GPU's (the plan, the exchange and the gather are the
code under test) and must reproduce the single-rank oracle smoothing bit for
bit; the plan's send and receive lists are also checked against each other.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ITERS = 6


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    sys.path.insert(0, ROOT)
    from multigpuegtsmoothing_b200 import datagen
    from oracle import pyoracle
    xyz = datagen.superquadrics(12000, seed=81)
    r = pyoracle.knn(xyz, 16)
    lists = pyoracle.egt(r["pos"], r["lists"], 0.65)
    valid = lists >= 0
    off = np.zeros(lists.shape[0] + 1, np.int64)
    off[1:] = np.cumsum(valid.sum(1))
    col = lists[valid].astype(np.int64)
    pos4 = np.zeros((lists.shape[0], 4), np.float32)
    pos4[:, :3] = r["pos"].T
    pos4[:, 3] = np.arange(lists.shape[0], dtype=np.float32)  # w rides along unchanged
    return r["pos"], lists, off, col, pos4


def _oracle_halfstep(pos_in, pos_out, off, col, rows, scale):
    from oracle import pyoracle
    pos_out.copy_(__import__("torch").from_numpy(
        pyoracle.taubin_rows_f32(pos_in.numpy(), rows, off.numpy(), col.numpy(), scale)))


def _rank_main(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from multigpuegtsmoothing_b200.sharded import ShardedTaubin, ShardPlan
    dist.init_process_group("gloo", rank=rank, world_size=world)
    _, _, off, col, pos4 = _problem()
    plan = ShardPlan(off, col, world, rank)
    sm = ShardedTaubin(torch.from_numpy(pos4), plan, halfstep=_oracle_halfstep)
    sm.run(ITERS)
    full = sm.gather()
    out[rank] = (full.numpy().copy(), plan.recv, [s.tolist() for s in plan.send], plan.halo.tolist(),
                 int(plan.lo), int(plan.hi))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_smoothing_equals_single_rank(world):
    out = mp.get_context("spawn").Manager().dict()
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    from oracle import pyoracle
    pos, lists, _, _, pos4 = _problem()
    want = pyoracle.taubin_f32(pos, lists, ITERS)          # (3, n), one rank
    for r in range(world):
        full = out[r][0]
        assert np.array_equal(full[:, :3].T, want), r
        assert np.array_equal(full[:, 3], pos4[:, 3]), r
    # what rank p receives from rank q is what q sends to p, element for element
    for p in range(world):
        _, recv, _, halo, _, _ = out[p]
        for q in range(world):
            if q == p:
                continue
            start, cnt = recv[q]
            qlo = out[q][4]
            sent = [qlo + i for i in out[q][2][p]]
            assert halo[start:start + cnt] == sent, (p, q)


def test_plan_single_rank_and_bounds():
    sys.path.insert(0, ROOT)
    from multigpuegtsmoothing_b200.sharded import ShardPlan
    _, _, off, col, _ = _problem()
    p = ShardPlan(off, col, 1, 0)
    assert p.halo.size == 0 and p.rows == off.shape[0] - 1
    assert np.array_equal(p.col, col.astype(np.int32))
    n = off.shape[0] - 1
    q = ShardPlan(off, col, 2, 1, bounds=np.array([0, 100, n]))
    assert (q.lo, q.hi) == (100, n)
    with pytest.raises(ValueError):
        ShardPlan(off, col, 2, 0, bounds=np.array([0, n + 1, n]))
