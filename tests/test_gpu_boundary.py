"""The KNNInterface drop-in boundary on the GPU.

* The reference's own consumers -- EGT_CUDA, Normal_CUDA and getOutputPoints,
  compiled unmodified from its sources against its KNNInterface.cuh -- run on
  this library's providers through egtb200::ReferenceView
  (oracle/ref/consumer_harness.cu) and must reproduce the reference's own run:
  EGT lists, smoothed positions, normals and output points.  This library's
  output stage, run between the reference's normals and output stages, reads
  what the reference's smoother left in the provider's slots.
* The threshold of GRIDCUDAKNNSELF_COMPACT(k, thres) at a finite value, set
  through egt_set_threshold, against the oracle's search with that threshold.
"""
import ctypes as C
import os

import numpy as np
import pytest

from golden_util import load
from multigpuegtsmoothing_b200 import datagen

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CONSUMER = os.path.join(ROOT, "oracle", "_ref", "libegtref_consumer.so")


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.fixture(scope="module")
def consumers(capi):
    if not os.path.exists(CONSUMER):
        pytest.skip("oracle/_ref/libegtref_consumer.so not built (needs the reference sources)")
    lib = C.CDLL(CONSUMER)
    lib.egtcons_cloud.restype = C.c_int
    lib.egtcons_cloud.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int] + [C.c_void_p] * 5
    lib.egtcons_mesh.restype = C.c_int
    lib.egtcons_mesh.argtypes = ([C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float]
                                 + [C.c_void_p] * 4)
    return lib


def test_reference_consumers_on_cloud_provider(consumers):
    d, m = load("ref_sphere_small")
    xyz = np.ascontiguousarray(d["in_xyz"], np.float32)
    n, k = xyz.shape[0], m["k"]
    knn = np.empty((n, k), np.int32)
    pos = np.empty((3, n), np.float32)
    nrm = np.empty((3, n), np.float32)
    out = np.empty((3, n), np.float32)
    out_lib = np.empty((3, n), np.float32)
    rc = consumers.egtcons_cloud(_p(xyz), n, k, m["iters"], m["alpha"], 1, _p(knn), _p(pos), _p(nrm), _p(out),
                                 _p(out_lib))
    assert rc == 0
    assert np.array_equal(knn, d["ref_knn_egt"])
    assert np.array_equal(pos, d["ref_pos_out"])
    assert np.array_equal(out, d["ref_out_xyz"])
    assert np.array_equal(out_lib, d["ref_out_xyz"])
    # the reference's normal code on the same positions and lists: its normals exactly
    assert np.array_equal(nrm, d["ref_normals"])


def test_reference_consumers_on_mesh_provider(consumers):
    d, m = load("ref_torus_small")
    xyz = np.ascontiguousarray(d["in_xyz"], np.float32)
    tris = np.ascontiguousarray(d["in_tris"], np.uint32)
    n, k = xyz.shape[0], m["k"]
    knn = np.empty((n, k), np.int32)
    pos = np.empty((3, n), np.float32)
    out = np.empty((3, n), np.float32)
    out_lib = np.empty((3, n), np.float32)
    rc = consumers.egtcons_mesh(_p(xyz), n, _p(tris), tris.shape[0], k, m["iters"], m["alpha"], _p(knn), _p(pos),
                                _p(out), _p(out_lib))
    assert rc == 0
    assert np.array_equal(knn, d["ref_knn_egt"])
    assert np.array_equal(pos, d["ref_pos_out"])
    assert np.array_equal(out, d["ref_out_xyz"])
    assert np.array_equal(out_lib, d["ref_out_xyz"])


@pytest.mark.parametrize("k,frac", [(16, 1.0), (40, 1.2)])
def test_finite_threshold_matches_oracle(capi, oracle, k, frac):
    """GRIDCUDAKNNSELF_COMPACT(k, thres) with thres a fraction of the typical
    k-th neighbour distance: admission is cut at thres, under-full lists continue
    while a face lies within sqrt(thres), so rows end short -- as the oracle's
    restatement of the reference does."""
    xyz = datagen.sphere_cloud(30000, 0.005, 71)
    r0 = oracle.knn(xyz, k)
    scale = float(r0["ext"][1]) - float(r0["ext"][0])
    kth = np.sqrt(r0["kth"][r0["lists"][:, 0] >= 0])
    thres = float(np.median(kth) * frac * scale)
    g = capi.GridStructure(xyz)
    g.GRIDCUDAKNNSELF_COMPACT(k, thres)
    r = oracle.knn(xyz, k, thres=thres)
    assert np.array_equal(g.sorted_lists(), r["lists"])
    assert g.timings()["invalid_queries"] == r["invalid"]
    short = (r["lists"] < 0).any(1).sum()  # rows cut short by the threshold
    assert 0 < short < xyz.shape[0]
    g.close()
