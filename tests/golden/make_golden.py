"""Generate the golden fixtures from the reference implementation itself.

Runs the UNMODIFIED reference (built from its own sources by oracle/ref/Makefile
into oracle/_ref/libegtref.so) on seeded synthetic inputs and stores what it
produced, so that the CPU oracle and the CUDA kernels can be pinned against the
reference without the reference being present.  Needs a GPU; run it on the
B200 box from the repository root:

    make -C oracle/ref && python tests/golden/make_golden.py --out tests/golden

Small cases are stored in full; the full-size configurations are stored as
SHA-256 digests of every output array plus a seeded sample of rows.  The inputs
are regenerated from their seeds (multigpuegtsmoothing_b200.datagen) and their
digest is stored too, so a change of generator is detected instead of being
mistaken for a parity failure.
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from multigpuegtsmoothing_b200 import datagen  # noqa: E402

LIB = os.path.join(ROOT, "oracle", "_ref", "libegtref.so")


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def load():
    lib = C.CDLL(LIB)
    lib.egtref_cloud.restype = C.c_int
    lib.egtref_cloud.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int] + [C.c_void_p] * 9
    lib.egtref_query.restype = C.c_int
    lib.egtref_query.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    lib.egtref_mesh.restype = C.c_int
    lib.egtref_mesh.argtypes = ([C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float]
                                + [C.c_void_p] * 8)
    return lib


def run_cloud(lib, xyz, k, iters, alpha, normals):
    n = xyz.shape[0]
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    o = dict(knn_raw=np.empty((n, k), np.int32), knn_egt=np.empty((n, k), np.int32),
             pos_in=np.empty((3, n), np.float32), pos_out=np.empty((3, n), np.float32),
             perm=np.empty(n, np.int32), extents=np.empty(2, np.float32),
             normals=np.empty((3, n), np.float32), out_xyz=np.empty((3, n), np.float32),
             stage_ms=np.empty(4, np.float32))
    rc = lib.egtref_cloud(_p(xyz), n, k, iters, alpha, int(normals), _p(o["knn_raw"]), _p(o["knn_egt"]),
                          _p(o["pos_in"]), _p(o["pos_out"]), _p(o["perm"]), _p(o["extents"]),
                          _p(o["normals"]), _p(o["out_xyz"]), _p(o["stage_ms"]))
    if rc != 0:
        raise RuntimeError("reference cloud run failed")
    if not normals:
        del o["normals"]
    return o


def run_mesh(lib, xyz, tris, k, iters, alpha):
    n = xyz.shape[0]
    t = tris.shape[0]
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    tris = np.ascontiguousarray(tris, dtype=np.uint32)
    o = dict(knn_raw=np.empty((n, k), np.int32), knn_egt=np.empty((n, k), np.int32),
             pos_in=np.empty((3, n), np.float32), pos_out=np.empty((3, n), np.float32),
             perm=np.empty(n, np.int32), extents=np.empty(2, np.float32),
             out_xyz=np.empty((3, n), np.float32), stage_ms=np.empty(4, np.float32))
    rc = lib.egtref_mesh(_p(xyz), n, _p(tris), t, k, iters, alpha, _p(o["knn_raw"]), _p(o["knn_egt"]),
                         _p(o["pos_in"]), _p(o["pos_out"]), _p(o["perm"]), _p(o["extents"]),
                         _p(o["out_xyz"]), _p(o["stage_ms"]))
    if rc != 0:
        raise RuntimeError("reference mesh run failed")
    return o


def run_query(lib, xyz, q, k):
    xyz = np.ascontiguousarray(xyz, np.float32)
    q = np.ascontiguousarray(q, np.float32)
    knn = np.empty((q.shape[0], k), np.int32)
    ms = np.zeros(1, np.float32)
    rc = lib.egtref_query(_p(xyz), xyz.shape[0], _p(q), q.shape[0], k, _p(knn), _p(ms))
    if rc != 0:
        raise RuntimeError("egtref_query failed")
    return dict(knn=knn, stage_ms=ms)


def query_points(xyz, seed):
    """Queries for the query-vs-reference kNN: jittered reference points (on
    the surface), uniform points in and around the reference cube (some
    outside it) and exact copies of reference points (distance 0)."""
    g = np.random.default_rng(seed)
    lo, hi = xyz.min(0), xyz.max(0)
    span = float((hi - lo).max())
    near = xyz[g.choice(xyz.shape[0], 1500, replace=False)] + g.normal(0, 0.01 * span, (1500, 3))
    box = lo - 0.15 * span + g.random((800, 3)) * (1.3 * span)
    same = xyz[g.choice(xyz.shape[0], 200, replace=False)]
    return np.concatenate([near, box, same]).astype(np.float32)


def lattice_cloud(side=16, dup_frac=0.0, seed=21):
    g = np.random.Generator(np.random.PCG64(seed))
    ax = np.arange(side, dtype=np.float32)
    p = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)
    p = p[g.permutation(len(p))]
    return np.ascontiguousarray(p, dtype=np.float32)


def with_duplicates(xyz, frac, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    n = xyz.shape[0]
    m = int(n * frac)
    src = g.integers(0, n, m)
    out = np.concatenate([xyz, xyz[src]])
    return np.ascontiguousarray(out[g.permutation(len(out))], dtype=np.float32)


def save_full(path, meta, inputs, outs):
    arrs = {f"in_{k}": v for k, v in inputs.items()}
    arrs.update({f"ref_{k}": v for k, v in outs.items()})
    arrs["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(path, **arrs)


def save_digest(path, meta, inputs, outs, rows=256, seed=99):
    g = np.random.Generator(np.random.PCG64(seed))
    arrs = {}
    digests = {f"in_{k}": sha(v) for k, v in inputs.items()}
    for k, v in outs.items():
        digests[f"ref_{k}"] = sha(v)
    n = outs["perm"].shape[0]
    pick = np.sort(g.choice(n, size=min(rows, n), replace=False)).astype(np.int64)
    arrs["rows"] = pick
    for k in ("knn_raw", "knn_egt"):
        arrs[f"ref_{k}_rows"] = outs[k][pick]
    for k in ("pos_in", "pos_out", "out_xyz", "normals"):
        if k in outs:
            arrs[f"ref_{k}_cols"] = outs[k][:, pick]
    arrs["ref_extents"] = outs["extents"]
    if n <= 200_000:
        arrs["ref_perm"] = outs["perm"]
    meta = dict(meta, digests=digests)
    arrs["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(path, **arrs)


MST_LIB = os.path.join(ROOT, "oracle", "_ref", "libegtref_mst.so")


def run_orient_kruskal(knn, nrm, k_use, xyz=None):
    """The reference's CPU orient_kruskal (MST.cpp:399-423), unmodified, on
    (n, k) lists and (3, n) normals; returns (normals, milliseconds)."""
    lib = C.CDLL(MST_LIB)
    f = lib.egtref_orient_kruskal
    f.restype = C.c_double
    f.argtypes = [C.c_void_p] * 7 + [C.c_int] * 3
    knn = np.ascontiguousarray(knn, dtype=np.int32)
    n, k = knn.shape
    out = np.array(nrm, dtype=np.float32, order="C", copy=True)
    pos = np.zeros((3, n), np.float32) if xyz is None else np.array(xyz, dtype=np.float32, order="C", copy=True)
    ms = f(_p(knn), _p(out[0]), _p(out[1]), _p(out[2]), _p(pos[0]), _p(pos[1]), _p(pos[2]), n, k, int(k_use))
    return out, ms


def orient_cases():
    """Inputs for the CPU-orienter fixtures: oracle kNN lists and unoriented
    oracle PCA normals with seeded random signs.  Built with the CPU oracle
    (oracle/pyoracle.py), which is test infrastructure like this script."""
    from oracle import pyoracle
    rng = np.random.default_rng(41)
    cases = []
    # a noisy sphere: one component, first 10 of 16 entries used
    kn = pyoracle.knn(datagen.sphere_cloud(20000, 0.005, 42), 16)
    nrm = pyoracle.normals(kn["pos"], kn["lists"])
    nrm *= np.where(rng.random(nrm.shape[1]) < 0.5, -1.0, 1.0).astype(np.float32)
    cases.append(("ref_orient_sphere.npz", "sphere_cloud(20000,0.005,42) k=16 oracle lists and PCA normals, random signs",
                  kn["lists"], nrm, 10))
    # two clouds that share no list edge, 20% of the entries blanked (-1, as the
    # EGT filter leaves them), and five rows with no neighbours: several trees
    a = pyoracle.knn(datagen.sphere_cloud(6000, 0.005, 43), 12)
    b = pyoracle.knn(datagen.sphere_cloud(3000, 0.01, 44), 12)
    lists = np.concatenate([a["lists"], np.where(b["lists"] >= 0, b["lists"] + 6000, -1),
                            np.full((5, 12), -1, np.int32)]).astype(np.int32)
    lists[rng.random(lists.shape) < 0.2] = -1
    nrm = np.concatenate([pyoracle.normals(a["pos"], a["lists"]), pyoracle.normals(b["pos"], b["lists"]),
                          np.tile(np.array([[0.0], [0.0], [1.0]], np.float32), (1, 5))], axis=1)
    nrm *= np.where(rng.random(nrm.shape[1]) < 0.5, -1.0, 1.0).astype(np.float32)
    cases.append(("ref_orient_forest.npz", "sphere_cloud(6000,0.005,43) + sphere_cloud(3000,0.01,44) k=12, "
                  "20% of entries blanked, 5 empty rows; random signs", lists, nrm, 12))
    # a lattice with every normal (0, 0, +-1): every weight is exactly 0, so
    # the order is (u, v) alone and union-by-rank ties decide the roots
    kn = pyoracle.knn(lattice_cloud(24), 8)
    n = kn["lists"].shape[0]
    nrm = np.zeros((3, n), np.float32)
    nrm[2] = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    cases.append(("ref_orient_ties.npz", "lattice_cloud(24) k=8 oracle lists, normals (0,0,+-1)", kn["lists"], nrm, 8))
    # axis-aligned normals: dot products are exactly +-1 or exactly 0, so the
    # trees cross edges whose dot product is zero, where the walk leaves the
    # child's sign as it is
    kn = pyoracle.knn(lattice_cloud(20, seed=45), 6)
    n = kn["lists"].shape[0]
    nrm = np.zeros((3, n), np.float32)
    nrm[rng.integers(0, 3, n), np.arange(n)] = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    cases.append(("ref_orient_zero.npz", "lattice_cloud(20,seed=45) k=6 oracle lists, random axis normals +-e_x/e_y/e_z",
                  kn["lists"], nrm, 6))
    return cases


def make_orient(out_dir, timings):
    for name, gen, lists, nrm, k_use in orient_cases():
        o, ms = run_orient_kruskal(lists, nrm, k_use)
        timings[name[:-4]] = ms
        save_full(os.path.join(out_dir, name), dict(kind="orient_kruskal", gen=gen, k_use=int(k_use)),
                  {"knn": lists, "nrm_in": nrm}, {"nrm_out": o})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--big", action="store_true", help="also run the 4M-point timing case")
    ap.add_argument("--only-query", action="store_true", help="only the query-vs-reference kNN fixtures")
    ap.add_argument("--only-orient", action="store_true",
                    help="only the CPU-orienter fixtures (MST.cpp; needs no GPU)")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.only_orient:
        t = {}
        make_orient(a.out, t)
        print(json.dumps(t))
        return
    lib = load()
    timings = {}

    # query-vs-reference kNN (GRIDCUDAKNNCompact): a noisy sphere and a lattice (ties)
    xyz = datagen.sphere_cloud(8000, 0.005, 31)
    q = query_points(xyz, 32)
    o = run_query(lib, xyz, q, 16)
    save_full(os.path.join(a.out, "ref_query_sphere.npz"),
              dict(kind="query", gen="sphere_cloud(8000,0.005,31); query_points(xyz,32)", k=16),
              {"xyz": xyz, "queries": q}, {"knn": o["knn"]})
    xyz = lattice_cloud(12)
    t = np.arange(-2, 14, dtype=np.float32) * np.float32(0.5)
    q = np.stack(np.meshgrid(t, t, t, indexing="ij"), -1).reshape(-1, 3)[::7].copy()
    o = run_query(lib, xyz, q, 20)
    save_full(os.path.join(a.out, "ref_query_lattice.npz"),
              dict(kind="query", gen="lattice_cloud(12); half-step lattice queries [-1, 6.5]^3 every 7th", k=20),
              {"xyz": xyz, "queries": q}, {"knn": o["knn"]})
    if a.only_query:
        return

    # 1. small noisy sphere, full arrays, with normals
    xyz = datagen.sphere_cloud(4096, 0.005, 11)
    meta = dict(kind="cloud", gen="sphere_cloud(4096,0.005,11)", k=16, iters=10, alpha=0.65, normals=True)
    o = run_cloud(lib, xyz, 16, 10, 0.65, True)
    timings["sphere_small"] = o.pop("stage_ms").tolist()
    save_full(os.path.join(a.out, "ref_sphere_small.npz"), meta, {"xyz": xyz}, o)

    # 2. lattice (exact distance ties everywhere), kNN + EGT + a few Taubin steps
    xyz = lattice_cloud(16)
    meta = dict(kind="cloud", gen="lattice_cloud(16)", k=26, iters=4, alpha=0.65, normals=False)
    o = run_cloud(lib, xyz, 26, 4, 0.65, False)
    timings["lattice"] = o.pop("stage_ms").tolist()
    save_full(os.path.join(a.out, "ref_lattice.npz"), meta, {"xyz": xyz}, o)

    # 3. sphere with 10% exact duplicates (zero distances, self-exclusion by index)
    xyz = with_duplicates(datagen.sphere_cloud(3000, 0.005, 12), 0.1, 13)
    meta = dict(kind="cloud", gen="with_duplicates(sphere_cloud(3000,0.005,12),0.1,13)", k=12, iters=3,
                alpha=0.65, normals=False)
    o = run_cloud(lib, xyz, 12, 3, 0.65, False)
    timings["dups"] = o.pop("stage_ms").tolist()
    save_full(os.path.join(a.out, "ref_dups.npz"), meta, {"xyz": xyz}, o)

    # 4. small torus mesh, full arrays
    xyz, tris = datagen.torus_mesh(64, 32, seed=14)
    meta = dict(kind="mesh", gen="torus_mesh(64,32,seed=14)", k=40, iters=10, alpha=1e-8)
    o = run_mesh(lib, xyz, tris, 40, 10, 1e-8)
    timings["torus_small"] = o.pop("stage_ms").tolist()
    save_full(os.path.join(a.out, "ref_torus_small.npz"), meta, {"xyz": xyz, "tris": tris}, o)

    # 5. full-size sphere cloud (35,947 points, k=40, 150 iterations): digests + samples
    xyz = datagen.sphere_cloud()
    meta = dict(kind="cloud", gen="sphere_cloud()", k=40, iters=150, alpha=0.65, normals=True)
    o = run_cloud(lib, xyz, 40, 150, 0.65, True)
    timings["sphere_c1"] = o.pop("stage_ms").tolist()
    save_digest(os.path.join(a.out, "ref_sphere_c1.npz"), meta, {"xyz": xyz}, o)

    # 6. full-size torus mesh (131,072 vertices, 262,144 triangles): digests + samples
    xyz, tris = datagen.torus_mesh()
    meta = dict(kind="mesh", gen="torus_mesh()", k=40, iters=150, alpha=1e-8)
    o = run_mesh(lib, xyz, tris, 40, 150, 1e-8)
    timings["torus_c2"] = o.pop("stage_ms").tolist()
    save_digest(os.path.join(a.out, "ref_torus_c2.npz"), meta, {"xyz": xyz, "tris": tris}, o)

    if a.big:
        xyz = datagen.superquadrics()
        t0 = time.time()
        o = run_cloud(lib, xyz, 40, 300, 0.65, False)
        timings["superquadrics_4m"] = o.pop("stage_ms").tolist()
        timings["superquadrics_4m_wall_s"] = time.time() - t0
        save_digest(os.path.join(a.out, "ref_superquadrics_4m.npz"),
                    dict(kind="cloud", gen="superquadrics()", k=40, iters=300, alpha=0.65, normals=False),
                    {"xyz": xyz}, o, rows=1024)
    with open(os.path.join(a.out, "ref_timings.json"), "w") as f:
        json.dump(timings, f, indent=1)
    print(json.dumps(timings))


if __name__ == "__main__":
    main()
