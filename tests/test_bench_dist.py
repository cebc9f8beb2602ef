"""The multi-rank plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1.

`bench.py --gpus N` runs one replica of the workload per rank (the queries
shard with no exchange), takes every time as the maximum over ranks and
reports the whole-job rate.  These tests run that plumbing with world size 2
without a GPU, and the reference arm under torch.distributed.run, where rank
0 alone measures and prints its line.
"""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup()
    assert (w, r) == (world, rank) and dist.get_backend() == "gloo"
    bench.barrier(w)
    slowest = bench.max_over_ranks(w, 10.0 + rank)        # the per-rank step time, ms
    rate = bench.aggregate_rate(w, 1000.0, slowest * 1e-3)  # 1000 units per rank
    out[rank] = (slowest, rate)
    dist.destroy_process_group()


def test_max_over_ranks_and_rate_two_gloo_ranks():
    out = mp.Manager().dict()
    mp.spawn(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True)
    for rank in (0, 1):
        slowest, rate = out[rank]
        assert slowest == 11.0                        # every rank sees the slowest rank's time
        assert abs(rate - 2 * 1000.0 / 0.011) < 1e-6  # all ranks' units over that time


def test_reference_arm_under_torchrun_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--points", "20000", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout  # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["config"]["n_points"] == 20000
    assert d["e2e"]["h2d_bytes_per_step"] == 0


def test_fp32_rates_and_clock_fallback():
    """The FP32 rate report: operations = evaluations x operations each, over
    the stage time, against 148 SMs x 128 lanes x 2 at the sampled clock; and
    the clock sampler reports what it could not sample instead of failing."""
    sys.path.insert(0, ROOT)
    import bench
    r = bench.fp32_rates(10 ** 9, 10.0, 2 * 10 ** 9, 20.0, {"sm_mhz": 1000.0})
    assert abs(r["knn"]["achieved"] - 0.8) < 1e-9  # 1e9 * 8 / 10 ms = 0.8 TFLOP/s
    assert abs(r["egt"]["achieved"] - 2.4) < 1e-9  # 2e9 * 24 / 20 ms
    assert abs(r["knn"]["peak"] - 148 * 128 * 2 * 1e9 / 1e12) < 1e-9
    assert r["knn"]["frac"] == r["knn"]["achieved"] / r["knn"]["peak"]
    # no clock sample: the peak falls back to the nominal maximum clock
    assert abs(bench.fp32_rates(1, 1.0, 1, 1.0, {"sm_mhz": None})["knn"]["peak"] - 148 * 128 * 2 * 1.965e9 / 1e12) < 1e-9
    clk = bench.ClockSampler(0).stop()
    assert set(("sm_mhz", "sm_max_mhz", "reasons")) <= set(clk)
