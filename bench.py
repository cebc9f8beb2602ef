"""Benchmark: grid kNN (k=40) Mqueries/s and Taubin iterations/s at 4M points.

Workload (one step): the 4,000,000-point superquadric cloud with a 50:1
clustered density (multigpuegtsmoothing_b200.datagen.superquadrics, seed 3) --
normalisation, cell sort and hierarchy build, then the exact k=40 grid kNN
(the reference's GridStructure + GRIDCUDAKNNSELF_COMPACT semantics; the
cell-tile search, egt_knn's default, unless --knn-mode says otherwise).  `value`
is queries per second over the whole step with the points already in HBM;
`e2e` is the same through the C ABI from pinned host memory (H2D of the
points, provider creation, kNN, D2H of the n*k neighbour ids in original
order).  The Taubin loop (EGT filter, then 300 lambda/mu iterations in one
CUDA graph) is timed in the same run and reported as taubin_iters_per_s with
its own HBM roofline, followed by the normals and their orientation.  Rank 0
also compares the proposal-driven kNN with the plain grid kNN on the 20M-point
k=64 sheets workload (learned_vs_plain; --no-learned skips it) and runs the
256-cloud batched workload (batched; --no-batched skips it).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun (N > 1) every rank runs its own replica of the workload (weak
scaling, no collective on the data path); times are the max over ranks.
`--impl reference` times the reference algorithm's CPU restatement on the
host cores on a bounded sample of the same workload (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS = 4_000_000
KNN_MODES = {"plain": 0, "select": 2, "tile": 3}  # egt_config.knn_mode: EGT_KNN_PLAIN, _SELECT, _TILE
K = 40
ITERS = 300
ALPHA = 0.65
SEED = 3


def load_points(n=N_POINTS, seed=SEED):
    from multigpuegtsmoothing_b200 import datagen
    cache = os.path.join(tempfile.gettempdir(), f"egt_bench_superquadrics_{n}_{seed}.npy")
    if os.path.exists(cache):
        try:
            return np.load(cache)
        except Exception:
            pass
    xyz = datagen.superquadrics(n, seed=seed)
    try:
        np.save(cache, xyz)
    except OSError:
        pass
    return xyz


def profiled_traffic(kernel: str):
    """DRAM bytes (read + write) per launch of `kernel` at the bench workload,
    from the committed ncu summary (one capture of dram__bytes_read.sum and
    dram__bytes_write.sum); None when no capture is recorded."""
    import re
    p = os.path.join(ROOT, "profiles", "dram_traffic_superquadrics_4m.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        m = re.match(r"\|\s*`" + re.escape(kernel) + r"`\s*\|.*\|\s*([0-9]+)\s*\|\s*$", line)
        if m:
            return int(m.group(1))
    return None


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every 10 ms from a background thread (the region can
    be shorter than nvidia-smi's 200 ms loop), nvidia-smi when NVML is absent.
    Reads only; changes no setting."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        import threading
        self.sm, self.smax, self.reasons = [], [], set()
        self.p = None
        self.thread = None
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        nvml_index = int(ids[index]) if index < len(ids) and ids[index].isdigit() else index
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(nvml_index)
            self.masks = (pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                          pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap)
        except Exception:
            self.nvml = None
        if self.nvml is not None:
            self.stop_flag = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(nvml_index), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def _sample(self, with_max: bool = False):
        # the maximum clock is a constant: read at the start and the end only
        # (each NVML query can take milliseconds)
        nv = self.nvml
        self.sm.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
        if with_max:
            self.smax.append(float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)))
        active = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        for nm, m in zip(self.NAMES, self.masks):
            if active & m:
                self.reasons.add(nm)

    def _poll(self):
        first = True
        while True:
            try:
                self._sample(with_max=first)
            except Exception:
                return
            first = False
            if self.stop_flag.wait(0.01):
                return

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join()
            try:
                self._sample(with_max=True)  # at least one sample at the end of the region
            except Exception:
                pass
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
            return {"sm_mhz": statistics.median(self.sm) if self.sm else None,
                    "sm_max_mhz": max(self.smax) if self.smax else None,
                    "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "nvml, 10 ms"}
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        for r in rows:
            try:
                self.sm.append(float(r[1]))
                self.smax.append(float(r[2]))
                for nm, v in zip(self.NAMES, r[5:9]):
                    if v.strip().lower() == "active":
                        self.reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None,
                "sm_max_mhz": max(self.smax) if self.smax else None,
                "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "nvidia-smi, 200 ms"}


def fp32_rates(knn_evals, knn_ms, egt_tests, egt_ms, clk):
    """kNN and EGT as FP32 operation rates from the counted evaluations: a
    candidate distance is 3 subtractions, 1 multiply and 2 fused multiply-adds
    (8 operations); an ellipsoid test is three 3-term affine transforms (6 each)
    and the quadratic form (6).  Peak: 148 SMs x 128 FP32 lanes x 2 operations
    per FMA at the SM clock sampled during the timed region (nominal, not
    measured)."""
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
    peak = 148 * 128 * 2 * mhz * 1e6 / 1e12

    def one(count, per, ms, what):
        achieved = count * per / (ms * 1e-3) / 1e12 if ms > 0 else 0.0
        return {"evaluations": int(count), "ops_per_evaluation": per, "what": what, "ms": ms,
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_kind": f"nominal FP32 at {mhz:.0f} MHz"}

    return {"knn": one(knn_evals, 8, knn_ms, "candidate (query, point) pairs of the kNN search, timed step "
                                             "(the cell-tile search computes each pair twice, counted once)"),
            "egt": one(egt_tests, 24, egt_ms, "ellipsoid tests (k_egt)")}


def dist_setup(init: bool = True):
    """Rank, world size and local rank from the torchrun environment; with
    init and more than one rank, joins the process group (NCCL with one GPU per
    rank, gloo when no GPU is present)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and init:
        import datetime
        import torch
        import torch.distributed as dist
        timeout = datetime.timedelta(seconds=600)
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timeout, device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=timeout)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, v: float) -> float:
    """The largest of the ranks' values (every rank calls it, in the same order)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, units_per_rank: float, seconds: float) -> float:
    """Whole-job rate: every rank processes units_per_rank in the time of the
    slowest rank (weak scaling, replicas of the workload)."""
    return world * units_per_rank / seconds


def cpu_baseline(xyz, k, budget_s=20.0):
    """Oracle (CPU restatement of the reference algorithm) on the host cores."""
    from oracle import pyoracle
    threads = pyoracle.num_threads()
    stride = 16
    tb, tq = pyoracle.knn_timed(xyz, k, stride)
    # grow the sample while it stays inside the budget
    while stride > 1 and tb + tq * 2 < budget_s / 2:
        stride //= 2
        tb, tq = pyoracle.knn_timed(xyz, k, stride)
    n = xyz.shape[0]
    est = tb + tq * stride  # all n queries
    return {"value": n / est / 1e6, "unit": "Mqueries/s", "cores": threads, "kind": "port",
            "sample": f"full grid build on {n} points + every {stride}th query "
                      f"({(n + stride - 1) // stride} queries), scaled to {n} queries",
            "build_s": tb, "query_s_sample": tq}


def cpu_stages(pos, knn_lists, egt_lists, smoothed, alpha, iters, taubin_sample_iters=2):
    """The later stages of the oracle on the host cores, on the inputs the GPU
    pipeline gives each stage (sorted space): the EGT filter over every row,
    Taubin for `taubin_sample_iters` iterations scaled to `iters`, the FP32
    normals and the spanning-forest orientation over every point."""
    from oracle import pyoracle
    out = {"cores": pyoracle.num_threads(), "kind": "port"}
    t = time.perf_counter()
    pyoracle.egt(pos, knn_lists, alpha)
    out["egt_filter_ms"] = (time.perf_counter() - t) * 1e3
    t = time.perf_counter()
    pyoracle.taubin_f32(pos, egt_lists, taubin_sample_iters)
    out[f"taubin_{iters}_iters_ms"] = (time.perf_counter() - t) * 1e3 * iters / taubin_sample_iters
    t = time.perf_counter()
    nrm = pyoracle.normals(smoothed, egt_lists, False)
    out["normals_ms"] = (time.perf_counter() - t) * 1e3
    t = time.perf_counter()
    pyoracle.orient(nrm, egt_lists)
    out["orientation_ms"] = (time.perf_counter() - t) * 1e3
    out["sample"] = (f"every row of the {pos.shape[1]}-point workload; Taubin {taubin_sample_iters} iterations "
                     f"scaled to {iters}")
    return out


def reference_gpu_stages():
    """The unmodified reference's per-stage GPU times, as tests/golden/time_reference.py
    last measured them on a B200 (None when the file is absent)."""
    p = os.path.join(ROOT, "tests", "golden", "ref_gpu_stages.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    d["source"] = "tests/golden/time_reference.py (unmodified reference built for sm_100a by oracle/ref/Makefile)"
    return d


def run_reference(args, world, rank):
    if rank != 0:
        return
    xyz = load_points(args.points)
    vals = []
    info = None
    for i in range(args.warmup + args.steps):
        info = cpu_baseline(xyz, K, budget_s=12.0)
        if i >= args.warmup:
            vals.append(info["value"])
    v = statistics.median(vals)
    line = {"metric": "Mqueries/s kNN (k=40) + Taubin iters/s at 4M pts; learned vs plain, exact",
            "value": v, "unit": "Mqueries/s", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"superquadrics {xyz.shape[0]} points, 50:1 clustered density, k=40 exact grid kNN",
                       "n_points": int(xyz.shape[0]), "k": K},
            "cpu_baseline": dict(info, value=v),
            "e2e": {"value": v, "unit": "Mqueries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def learned_compare(capi, xyz, k, train, workload):
    """Trains a proposal network on the clouds `train` with the device's own
    training kernels, tunes its class threshold by timing, then times on xyz
    the plain grid kNN (egt_knn's default ring search), the proposal-driven kNN
    and the block-selection search (best of 3 each, CUDA events around the
    search, the proposal's features and network included), and compares their
    lists for identity."""
    p = capi.SearchProposal(k, seed=1)
    for pts in train:
        gt = capi.GridStructure(pts)
        gt.GRIDCUDAKNNSELF_COMPACT(k)
        p.collect(gt)
        gt.close()
    losses = p.train(3000)
    g = capi.GridStructure(xyz, config=capi.default_config(knn_mode=KNN_MODES["plain"]))
    g.GRIDCUDAKNNSELF_COMPACT(k)
    ref = g.sorted_lists()
    p.tune(g)
    sel = capi.GridStructure(xyz, config=capi.default_config(knn_mode=KNN_MODES["select"]))
    til = capi.GridStructure(xyz, config=capi.default_config(knn_mode=KNN_MODES["tile"]))
    plain_ms, learned_ms, select_ms, tile_ms = [], [], [], []
    for _ in range(3):
        g.GRIDCUDAKNNSELF_COMPACT(k)
        plain_ms.append(g.timings()["knn_ms"])
        g.GRIDCUDAKNNSELF_LEARNED(k, p)
        learned_ms.append(g.timings()["knn_ms"])
        t = g.timings()
        sel.GRIDCUDAKNNSELF_COMPACT(k)
        select_ms.append(sel.timings()["knn_ms"])
        til.GRIDCUDAKNNSELF_COMPACT(k)
        tile_ms.append(til.timings()["knn_ms"])
    same = all(bool(np.array_equal(x.sorted_lists(), ref)) for x in (g, sel, til))
    sel.close()
    til.close()
    n = xyz.shape[0]
    out = {"workload": workload,
           "plain": "EGT_KNN_PLAIN: the reference's ring expansion (k_knn_plain)",
           "plain_ms": min(plain_ms), "learned_ms": min(learned_ms),
           "plain_mqueries_s": n / min(plain_ms) / 1e3, "learned_mqueries_s": n / min(learned_ms) / 1e3,
           "speedup": min(plain_ms) / min(learned_ms), "lists_identical": same, "tau": p.tau,
           "box_queries_frac": t["box_queries"] / n, "certified_frac": t["certified_queries"] / n,
           "train_loss_first_last": [float(losses[0]), float(losses[-1])],
           "block_selection_ms": min(select_ms), "block_selection_mqueries_s": n / min(select_ms) / 1e3,
           "block_selection_note": "the block-selection search (EGT_KNN_SELECT) on the same cloud, same lists",
           "tile_ms": min(tile_ms), "tile_mqueries_s": n / min(tile_ms) / 1e3,
           "tile_note": "the cell-tile search (EGT_KNN_TILE, egt_knn's default; the ring search for k outside "
                        "16..64) on the same cloud, same lists"}
    g.close()
    p.close()
    return out


def learned_vs_plain(capi):
    """The learned-proposal workload: 20M points on Gaussian-thickened planar
    and spherical sheets with a 1000:1 density range, k=64, the network trained
    on two 2M-point clouds of the same generator (seeds 100, 101)."""
    from multigpuegtsmoothing_b200 import datagen
    k = 64
    cache = os.path.join(tempfile.gettempdir(), "egt_bench_sheets_20000000_5.npy")
    try:
        xyz = np.load(cache)
    except (OSError, ValueError):
        xyz = datagen.sheets(20_000_000, seed=5)
        try:
            np.save(cache, xyz)
        except OSError:
            pass
    train = [datagen.sheets(2_000_000, seed=s) for s in (100, 101)]
    return learned_compare(capi, xyz, k, train, f"sheets {xyz.shape[0]} points, 1000:1 density range, k={k}")


def learned_on_headline(capi, xyz):
    """The same comparison on the headline workload (the 4M-point superquadric
    cloud, k=40), the network trained on two 2M-point superquadric clouds of
    other seeds (100, 101)."""
    from multigpuegtsmoothing_b200 import datagen
    train = [datagen.superquadrics(2_000_000, seed=s) for s in (100, 101)]
    return learned_compare(capi, xyz, K, train,
                           f"superquadrics {xyz.shape[0]} points, 50:1 clustered density, k={K}")


def batched(capi, iters: int = 150, alpha: float = 0.65):
    """The batched workload: 256 clouds (noisy spheres and tori) with point
    counts log-uniform in 2K-500K and k drawn from {10, 20, 40}, seed 4, run
    through grid build, kNN, EGT filter and `iters` Taubin iterations with one
    launch per stage (egt_batch_run).  The first run autotunes the work chunk
    and the Taubin kernel; the best of 3 further runs is reported, stage by
    stage (CUDA events).  Four sampled clouds are checked against their own
    single-cloud pipeline, bit for bit."""
    from multigpuegtsmoothing_b200 import datagen
    clouds = datagen.batch_clouds(count=256, nmin=2000, nmax=500_000, seed=4)
    b = capi.Batch(clouds)
    b.run(iters, alpha=alpha)
    best = None
    for _ in range(3):
        b.run(iters, alpha=alpha)
        t = b.timings()
        total = t["grid_ms"] + t["knn_ms"] + t["egt_ms"] + t["taubin_ms"]
        if best is None or total < best[0]:
            best = (total, t)
    total, t = best
    out = b.output()
    sample = np.random.default_rng(4).choice(len(clouds), 4, replace=False)
    same = 0
    for c in sample:
        xyz, k = clouds[c]
        g = capi.GridStructure(xyz)
        g.GRIDCUDAKNNSELF_COMPACT(k)
        e = capi.EGT_CUDA(g)
        e.Filter(alpha)
        e.Taubin(iters)
        x, y, z = capi.getOutputPoints(g)
        g.close()
        same += bool(np.array_equal(out[c], np.stack([x, y, z], 1)))
    b.close()
    n = int(t["points"])
    return {"workload": f"{len(clouds)} clouds, 2K-500K points log-uniform, k in {{10,20,40}}, "
                        f"EGT + {iters} Taubin iterations (kNN + EGT in one fused launch or two, autotuned)",
            "points": n, "grid_ms": t["grid_ms"], "knn_ms": t["knn_ms"], "egt_ms": t["egt_ms"],
            "taubin_ms": t["taubin_ms"], "total_ms": total, "knn_mqueries_s": n / t["knn_ms"] / 1e3,
            "taubin_point_iters_per_s": n * iters / (t["taubin_ms"] * 1e-3),
            "clouds_bit_identical_to_single": f"{same}/{len(sample)}",
            "knn_chunk": t["knn_chunk"], "taubin_mode": t["taubin_mode"],
            "knn_egt_fused": bool(t["fused"]),
            "autotune_knn_egt_ms": {"one_fused_launch": t["fused_ms"], "two_launches": t["separate_ms"],
                                    "note": "kNN + EGT filter + CSR, measured by the autotuner; the faster runs"}}


def pipeline_configs(capi):
    """Stage times of this build on the two small single-cloud workloads, the
    35,947-point noisy sphere (k=40, alpha 0.65, 150 iterations, normals) and
    the 131,072-vertex torus mesh (1-ring capped at 40, alpha 1e-8, 150
    iterations): each pipeline runs once to warm up, then once timed (CUDA
    events per stage, egt_get_timings)."""
    from multigpuegtsmoothing_b200 import datagen
    out = {}
    sphere = datagen.sphere_cloud()
    xyz_t, tris = datagen.torus_mesh()
    for name in ("sphere_c1", "torus_c2"):
        for rep in range(2):
            if name == "sphere_c1":
                g = capi.GridStructure(sphere)
                g.GRIDCUDAKNNSELF_COMPACT(40)
                capi.EGT_CUDA(g).PerformSmoothing(150, 0.63, -0.64, 0.65)
                capi.Normal_CUDA(g).GetNormals()
            else:
                g = capi.GridMeshCuda(xyz_t, tris)
                g.GetNeighborsFromTriangles(40)
                capi.EGT_CUDA(g).PerformSmoothing(150, 0.63, -0.64, 1e-8)
            capi.getOutputPoints(g)
            t = g.timings()
            g.close()
        rec = {"points": int(t.get("points", 0)) or (sphere.shape[0] if name == "sphere_c1" else xyz_t.shape[0]),
               "grid_knn_ms": t["grid_ms"] + t["knn_ms"], "egt_taubin_ms": t["egt_ms"] + t["taubin_ms"],
               "output_ms": t["output_ms"]}
        if name == "sphere_c1":
            rec["normals_orient_ms"] = t["normals_ms"] + t["orient_ms"]
        out[name] = rec
    return out


def run_b200(args, world, rank, local):
    import torch
    from multigpuegtsmoothing_b200 import capi

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    xyz = load_points(args.points)
    n = xyz.shape[0]
    xyz_dev = torch.from_numpy(xyz).to(dev).contiguous()
    torch.cuda.synchronize()
    g = capi.GridStructure(None, device_ptr=xyz_dev.data_ptr(), n=n,
                           config=capi.default_config(knn_mode=KNN_MODES[args.knn_mode]))

    def step():
        g.UpdatePointsDevice(xyz_dev.data_ptr())
        g.GRIDCUDAKNNSELF_COMPACT(K)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = capi.kernel_launches()
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        g.UpdatePointsDevice(xyz_dev.data_ptr())
        ev[i][1].record(stream)
        g.GRIDCUDAKNNSELF_COMPACT(K)
        ev[i][2].record(stream)
    t1.record(stream)
    # wait with short sleeps, so that the clock sampler's thread runs while
    # the timed steps execute (a blocking synchronize gives it no turn)
    while not t1.query():
        time.sleep(0.0005)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    launches = (capi.kernel_launches() - launches0) // args.steps
    ms = max_over_ranks(world, t0.elapsed_time(t1)) / args.steps
    build_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    knn_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in ev)
    value = aggregate_rate(world, n, ms * 1e-3) / 1e6
    tm = g.timings()

    # roofline of the dominant kernel (the kNN query kernel): algorithmic bytes
    # 24 + 4k per query (own point 12 B, amortised grid point 12 B, k ids)
    peak, peak_kind = peaks()
    knn_kernel = {"plain": "k_knn_plain", "select": "k_knn_select", "tile": "k_knn_tile"}[args.knn_mode]
    knn_bytes = n * (24 + 4 * K)
    knn_gbs = knn_bytes / (knn_ms * 1e-3) / 1e9

    # The rest of the pipeline -- EGT filter, ITERS lambda/mu iterations in one
    # CUDA graph, normals and their orientation -- runs once untimed (the
    # device memory pool grows to the pipeline's peak: first-use costs that a
    # long-running process pays once), then again from the original points,
    # timed stage by stage.
    egt = capi.EGT_CUDA(g)
    for warm in (True, False):
        g.UpdatePointsDevice(xyz_dev.data_ptr())
        g.GRIDCUDAKNNSELF_COMPACT(K)
        if not warm and rank == 0 and world == 1 and not args.no_cpu_baseline:
            knn_lists, start_pos = g.sorted_lists(), g.sorted_positions()
        egt.Filter(ALPHA)
        tmf = g.timings()
        if warm:
            egt.Taubin(ITERS)
            capi.Normal_CUDA(g).GetNormals()
    t_egt, t_egt_kernel = tmf["egt_ms"], tmf["egt_kernel_ms"]
    nnz = tmf["csr_nnz"]
    knn_evals, egt_tests = tm["knn_evaluations"], tmf["egt_tests"]
    # first Taubin call on this CSR: Morton relabelling, per-tile tables and the
    # graph capture of the 2*ITERS half-steps, then the replay
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    egt.Taubin(ITERS)
    torch.cuda.synchronize()
    taubin_first_wall_ms = (time.perf_counter() - w0) * 1e3
    taubin_first_dev_ms = g.timings()["taubin_ms"]
    spill = g.timings()
    torch.cuda.synchronize()
    ta, tb_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(1, min(args.steps, 3))
    ta.record(stream)
    for _ in range(reps):
        egt.Taubin(ITERS)
    tb_.record(stream)
    torch.cuda.synchronize()
    taubin_ms = max_over_ranks(world, ta.elapsed_time(tb_)) / reps
    mbar = nnz / n
    taubin_bytes = 2 * ITERS * n * (28 + 4 * mbar)
    taubin_gbs = taubin_bytes / (taubin_ms * 1e-3) / 1e9

    # normals (PCA, FP64 re-solve of near-degenerate gaps) + spanning-tree orientation
    capi.Normal_CUDA(g).GetNormals()
    tmn = g.timings()
    stages_cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        stages_cpu = cpu_stages(start_pos, knn_lists, g.sorted_lists(), g.sorted_positions(), ALPHA, ITERS)
        del knn_lists, start_pos
    configs = pipeline_configs(capi) if rank == 0 and not args.no_configs else None

    # e2e through the C ABI with pinned host buffers
    host_xyz = torch.from_numpy(xyz).pin_memory()
    host_knn = torch.empty((n, K), dtype=torch.int32).pin_memory()
    e2e_times = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        barrier(world)
        s = time.perf_counter()
        h2 = capi.GridStructure(host_xyz.numpy())
        h2.knn_host(K, out=host_knn.numpy())  # search + original-order lists to host, copies overlapped
        h2.close()
        e = time.perf_counter() - s
        if i >= args.warmup:
            e2e_times.append(max_over_ranks(world, e))
    e2e_s = statistics.mean(e2e_times)
    e2e_value = aggregate_rate(world, n, e2e_s) / 1e6

    if rank == 0:
        line = {
            "metric": "Mqueries/s kNN (k=40) + Taubin iters/s at 4M pts; learned vs plain, exact",
            "value": value, "unit": "Mqueries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"superquadrics {n} points, 50:1 clustered density, k=40 exact grid kNN",
                       "n_points": n, "k": K, "parallelism": f"replicas{world}", "search": args.knn_mode,
                       "l2": "per-step footprint > L2 (n*k*4 = 640 MB of lists written per step)"},
            "stages_ms": {"grid_build": build_ms, "knn_query": knn_ms, "egt_filter": t_egt,
                          "egt_filter_kernel": t_egt_kernel,
                          "taubin_300_iters": taubin_ms, "normals": tmn["normals_ms"],
                          "orientation": tmn["orient_ms"],
                          "note": "egt_filter..orientation: second pass of the pipeline on a warm memory pool"},
            "taubin_first_call": {"device_ms": taubin_first_dev_ms, "wall_ms": taubin_first_wall_ms,
                                  "note": "first egt_taubin on a new CSR: Morton relabelling, per-tile tables, "
                                          "graph capture, then the 300 iterations; taubin_300_iters replays the "
                                          "cached graph"},
            "taubin_iters_per_s": ITERS / (taubin_ms * 1e-3),
            "taubin_roofline": {"bound": "hbm", "achieved": taubin_gbs, "peak": peak, "unit": "GB/s",
                                "frac": taubin_gbs / peak, "peak_kind": peak_kind,
                                "bytes_model": "2*iters*n*(28+4*m), m = kept neighbours per point",
                                "m_mean": mbar, "traffic": profiled_traffic("k_taubin_tiles"),
                                "kernel": "k_taubin_tiles (one half-step)"},
            "roofline": {"bound": "hbm", "achieved": knn_gbs, "peak": peak, "unit": "GB/s", "frac": knn_gbs / peak,
                         "traffic": profiled_traffic(knn_kernel), "kernel": knn_kernel,
                         "peak_kind": peak_kind,
                         "bytes_model": "n*(24+4k)"},
            "e2e": {"value": e2e_value, "unit": "Mqueries/s", "h2d_bytes_per_step": int(xyz.nbytes),
                    "d2h_bytes_per_step": int(n * K * 4)},
            "fp32": fp32_rates(knn_evals, knn_ms, egt_tests, t_egt_kernel, clk),
            "gpu_launches": int(launches),
            "clocks": clk,
            "knn_stats": {"invalid_queries": tm["invalid_queries"], "levels_used": tm["levels_used"],
                          "ring_search_queries": tm["knn_fallback"], "exact_reruns": tm["exact_reruns"],
                          "note": "ring_search_queries: rows the cell tiles (or the block selection) did not "
                                  "take or could not certify (equal distances, a k-th ball beyond the block, "
                                  "...), searched by the reference's ring expansion"},
            "taubin_tiles": {"tiles": spill["taubin_tiles"], "spilled": spill["taubin_spill_tiles"]},
        }
        if configs is not None:
            line["configs"] = configs
        ref_gpu = reference_gpu_stages()
        if ref_gpu is not None:
            line["reference_gpu"] = ref_gpu
        if not args.no_learned:
            line["learned_vs_plain"] = learned_vs_plain(capi)
            line["learned_vs_plain_headline"] = learned_on_headline(capi, xyz)
        if not args.no_batched:
            line["batched"] = batched(capi)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(xyz, K)
            line["cpu_baseline"]["stages"] = stages_cpu
        print(json.dumps(line), flush=True)
    g.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-proposal comparison")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-clouds workload")
    ap.add_argument("--no-configs", action="store_true", help="skip the 36K-sphere and torus-mesh stage times")
    ap.add_argument("--knn-mode", default="tile", choices=sorted(KNN_MODES),
                    help="search of the timed step: tile (the cell-tile search, egt_knn's default), plain (the "
                         "reference's ring search) or select")
    ap.add_argument("--points", type=int, default=N_POINTS,
                    help="workload size override (profiling a smaller case of the same step)")
    args = ap.parse_args()
    # the reference arm runs on rank 0 alone and needs no process group
    world, rank, local = dist_setup(init=args.impl != "reference")
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_b200(args, world, rank, local)
    finally:
        if world > 1 and args.impl != "reference":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
