"""Loading helpers for the golden fixtures produced by tests/golden/make_golden.py."""
import hashlib
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FULL = ["ref_sphere_small", "ref_lattice", "ref_dups"]
MESH_FULL = ["ref_torus_small"]
ORIENT = ["ref_orient_sphere", "ref_orient_forest", "ref_orient_ties", "ref_orient_zero"]


def load(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(bytes(d["meta"]).decode())
    return d, meta


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def regen(meta):
    """Regenerates the input of a digest fixture from its generator string."""
    from multigpuegtsmoothing_b200 import datagen
    gen = meta["gen"]
    if gen == "sphere_cloud()":
        return datagen.sphere_cloud(), None
    if gen == "torus_mesh()":
        return datagen.torus_mesh()
    if gen == "superquadrics()":
        return datagen.superquadrics(), None
    raise KeyError(gen)


def bbox_diag(xyz):
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    return float(np.linalg.norm(xyz.max(0) - xyz.min(0)))
