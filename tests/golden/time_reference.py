"""Time the UNMODIFIED reference per stage on the GPU it runs on.

The reference (built from its own sources by oracle/ref/Makefile into
oracle/_ref/libegtref.so) runs the CLI's pipeline on the three single-cloud
workloads -- the 35,947-point noisy sphere (k=40, 150 iterations, normals on),
the 131,072-vertex torus mesh (k=40, 150 iterations) and the 4,000,000-point
superquadric cloud (k=40, 300 iterations, normals on) -- and its harness times
each stage with CUDA events and a device sync: grid build + kNN (provider
creation from host points included), EGT filter + Taubin, normals + their
orientation (Normal_CUDA::GetNormals), output gather.  Each workload runs
twice; the second run is reported (the first pays CUDA context and allocator
start-up).  Test infrastructure: bench.py reports the file this writes as the
reference's GPU bar.  Needs a GPU; run it from the repository root:

    make -C oracle/ref && python tests/golden/time_reference.py --out tests/golden/ref_gpu_stages.json
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from multigpuegtsmoothing_b200 import datagen  # noqa: E402

LIB = os.path.join(ROOT, "oracle", "_ref", "libegtref.so")
STAGES = ["grid_knn_ms", "egt_taubin_ms", "normals_orient_ms", "output_ms"]


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "ref_gpu_stages.json"))
    ap.add_argument("--skip-4m-normals", action="store_true")
    a = ap.parse_args()
    lib = C.CDLL(LIB)
    lib.egtref_cloud.restype = C.c_int
    lib.egtref_cloud.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int] + [C.c_void_p] * 9
    lib.egtref_mesh.restype = C.c_int
    lib.egtref_mesh.argtypes = ([C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float]
                                + [C.c_void_p] * 8)
    try:
        gpu = subprocess.run(["nvidia-smi", "--query-gpu=name", "--format=csv,noheader", "-i", "0"],
                             capture_output=True, text=True, timeout=30).stdout.strip()
    except (OSError, subprocess.TimeoutExpired):
        gpu = "unknown"
    out = {"what": "unmodified reference, per-stage CUDA-event times (ms), second of two runs",
           "gpu": gpu, "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()), "workloads": {}}
    cases = [("sphere_c1", "cloud", datagen.sphere_cloud(), None, 40, 150, 0.65, True),
             ("torus_c2", "mesh") + datagen.torus_mesh() + (40, 150, 1e-8, False),
             ("superquadrics_4m", "cloud", datagen.superquadrics(), None, 40, 300, 0.65, not a.skip_4m_normals)]
    for name, kind, xyz, tris, k, iters, alpha, normals in cases:
        xyz = np.ascontiguousarray(xyz, dtype=np.float32)
        n = xyz.shape[0]
        runs = []
        for _ in range(2):
            ms = np.zeros(4, np.float32)
            t0 = time.time()
            if kind == "cloud":
                rc = lib.egtref_cloud(_p(xyz), n, k, iters, alpha, int(normals), *([None] * 8), _p(ms))
            else:
                t = np.ascontiguousarray(tris, dtype=np.uint32)
                rc = lib.egtref_mesh(_p(xyz), n, _p(t), t.shape[0], k, iters, alpha, *([None] * 7), _p(ms))
            if rc != 0:
                raise RuntimeError(f"reference run failed on {name}")
            runs.append((ms.tolist(), time.time() - t0))
        ms, wall = runs[-1]
        rec = dict(zip(STAGES, ms))
        rec.update(points=n, k=k, iters=iters, normals=normals, wall_s=wall)
        out["workloads"][name] = rec
        print(name, json.dumps(rec), flush=True)
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
