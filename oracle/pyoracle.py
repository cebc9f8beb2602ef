"""ctypes binding of the CPU oracle (oracle/libegt_oracle.so).

ORACLE / TEST INFRASTRUCTURE: imported only by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg, as the checker.
The library is built by ``make -C oracle`` (or __graft_entry__.build()).
All functions take and return numpy arrays; positions are (3, n) float32 SoA in
cell-sorted order, lists are (n, k) int32 sorted-space neighbour indices.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libegt_oracle.so")
_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, i32, f32 = C.c_void_p, C.c_int, C.c_float
        L.orc_num_threads.restype = i32
        L.orc_extents.argtypes = [vp, i32, vp]
        L.orc_knn.restype = i32
        L.orc_knn.argtypes = [vp, i32, i32, f32, vp, vp, vp, vp, vp, vp, vp]
        L.orc_knn_query.restype = i32
        L.orc_knn_query.argtypes = [vp, i32, vp, i32, i32, f32, vp, vp]
        L.orc_mesh_1ring.argtypes = [vp, i32, vp, i32, i32, vp, vp, vp, vp]
        L.orc_egt.argtypes = [vp, i32, i32, vp, f32, vp]
        L.orc_taubin_f32.argtypes = [vp, i32, i32, vp, i32, f32, f32]
        L.orc_taubin_f64.argtypes = [vp, i32, i32, vp, i32, C.c_double, C.c_double]
        L.orc_taubin_rows_f32.argtypes = [vp, i32, i32, vp, vp, f32, vp]
        L.orc_normals.argtypes = [vp, i32, i32, vp, i32, vp]
        L.orc_normal_gaps.argtypes = [vp, i32, i32, vp, vp]
        L.orc_orient.restype = i32
        L.orc_orient.argtypes = [i32, i32, vp, vp, vp]
        L.orc_orient_kruskal.argtypes = [vp, C.c_int64, i32, i32, vp, vp, vp, i32]
        L.orc_output.argtypes = [vp, vp, vp, i32, vp]
        L.orc_bruteforce.argtypes = [vp, i32, i32, vp, vp]
        L.orc_select_check.argtypes = [vp, i32, i32, vp]
        L.orc_knn_timed.argtypes = [vp, i32, i32, i32, vp, vp]
        L.orc_proposal_data.restype = i32
        L.orc_proposal_data.argtypes = [vp, i32, i32, vp, vp]
        L.orc_knn_proposal.restype = i32
        L.orc_knn_proposal.argtypes = [vp, i32, i32, vp, vp, vp, vp, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def num_threads() -> int:
    return lib().orc_num_threads()


def knn(xyz: np.ndarray, k: int, thres: float = 1e8):
    """Reference grid kNN.  Returns dict(lists, pos, perm, ext, level, kth, invalid, visited)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    n = xyz.shape[0]
    lists = np.empty((n, k), np.int32)
    pos = np.empty((3, n), np.float32)
    perm = np.empty(n, np.int32)
    ext = np.empty(2, np.float32)
    level = np.empty(n, np.int32)
    kth = np.empty(n, np.float32)
    visited = C.c_longlong(0)
    inv = lib().orc_knn(_p(xyz), n, k, float(thres), _p(lists), _p(pos), _p(perm), _p(ext), _p(level), _p(kth),
                        C.byref(visited))
    return dict(lists=lists, pos=pos, perm=perm, ext=ext, level=level, kth=kth, invalid=inv,
                visited=visited.value)


def knn_query(xyz: np.ndarray, queries: np.ndarray, k: int, thres: float = 1e8, with_status: bool = False):
    """Reference query-vs-reference kNN (GRIDCUDAKNNCompact + GetKNNIndexes):
    (nq, k) original reference ids in original query order, and the invalid
    count; with_status adds the per-query status (0 valid, 1 oversized cell,
    2 still searching after the last level)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    q = np.ascontiguousarray(queries, dtype=np.float32)
    out = np.empty((q.shape[0], k), np.int32)
    st = np.empty(q.shape[0], np.int32)
    inv = lib().orc_knn_query(_p(xyz), xyz.shape[0], _p(q), q.shape[0], k, float(thres), _p(out), _p(st))
    return (out, inv, st) if with_status else (out, inv)


def mesh_1ring(xyz: np.ndarray, tris: np.ndarray, k: int):
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    tris = np.ascontiguousarray(tris, dtype=np.uint32)
    n = xyz.shape[0]
    lists = np.empty((n, k), np.int32)
    pos = np.empty((3, n), np.float32)
    perm = np.empty(n, np.int32)
    ext = np.empty(2, np.float32)
    lib().orc_mesh_1ring(_p(xyz), n, _p(tris), tris.shape[0], k, _p(lists), _p(pos), _p(perm), _p(ext))
    return dict(lists=lists, pos=pos, perm=perm, ext=ext)


def egt(pos: np.ndarray, lists: np.ndarray, alpha: float) -> np.ndarray:
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    lists = np.ascontiguousarray(lists, dtype=np.int32)
    n, k = lists.shape
    out = np.empty_like(lists)
    lib().orc_egt(_p(pos), n, k, _p(lists), float(alpha), _p(out))
    return out


def taubin_f32(pos: np.ndarray, lists: np.ndarray, iters: int, lam=0.63, mu=-0.64) -> np.ndarray:
    p = np.array(pos, dtype=np.float32, order="C", copy=True)
    lists = np.ascontiguousarray(lists, dtype=np.int32)
    n, k = lists.shape
    lib().orc_taubin_f32(_p(p), n, k, _p(lists), iters, lam, mu)
    return p


def taubin_rows_f32(pos4: np.ndarray, rows: int, off: np.ndarray, col: np.ndarray, scale: float) -> np.ndarray:
    """One FP32 half-step over rows [0, rows) of a CSR whose columns index the
    (m, 4) float32 positions pos4 (own position of row i = pos4[i]); returns
    the (rows, 4) new positions."""
    pos4 = np.ascontiguousarray(pos4, dtype=np.float32)
    off = np.ascontiguousarray(off, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    out = np.empty((rows, 4), np.float32)
    lib().orc_taubin_rows_f32(_p(pos4), pos4.shape[0], rows, _p(off), _p(col), float(scale), _p(out))
    return out


def taubin_f64(pos: np.ndarray, lists: np.ndarray, iters: int, lam=0.63, mu=-0.64) -> np.ndarray:
    p = np.array(pos, dtype=np.float64, order="C", copy=True)
    lists = np.ascontiguousarray(lists, dtype=np.int32)
    n, k = lists.shape
    lib().orc_taubin_f64(_p(p), n, k, _p(lists), iters, float(np.float32(lam)), float(np.float32(mu)))
    return p


def normals(pos: np.ndarray, lists: np.ndarray, f64: bool = False) -> np.ndarray:
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    lists = np.ascontiguousarray(lists, dtype=np.int32)
    n, k = lists.shape
    out = np.empty((3, n), np.float32)
    lib().orc_normals(_p(pos), n, k, _p(lists), int(f64), _p(out))
    return out


def normal_gaps(pos: np.ndarray, lists: np.ndarray) -> np.ndarray:
    """(l1 - l0) / l2 of each point's FP64 covariance (sorted space): ~0 where
    the normal is not defined."""
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    lists = np.ascontiguousarray(lists, dtype=np.int32)
    n, k = lists.shape
    gap = np.empty(n, np.float64)
    lib().orc_normal_gaps(_p(pos), n, k, _p(lists), _p(gap))
    return gap


def orient(nrm: np.ndarray, lists: np.ndarray):
    """Orient sorted-space normals in place order; returns (normals, parent, ncomp)."""
    lists = np.ascontiguousarray(lists, dtype=np.int32)
    n, k = lists.shape
    out = np.array(nrm, dtype=np.float32, order="C", copy=True)
    parent = np.empty(n, np.int32)
    nc = lib().orc_orient(n, k, _p(lists), _p(out), _p(parent))
    return out, parent, nc


def orient_kruskal(knn: np.ndarray, nrm: np.ndarray, k_use: int, key32: bool = False) -> np.ndarray:
    """The reference's CPU orienter orient_kruskal (MST.cpp:399-423) on
    (n, k) lists and (3, n) normals; returns the oriented (3, n) normals.
    key32 reproduces the reference's 32-bit edge key, which wraps around
    above 46,340 points (colliding pairs are then dropped)."""
    knn = np.ascontiguousarray(knn, dtype=np.int32)
    n, k = knn.shape
    out = np.array(nrm, dtype=np.float32, order="C", copy=True)
    lib().orc_orient_kruskal(_p(knn), n, k, int(k_use), _p(out[0]), _p(out[1]), _p(out[2]), int(key32))
    return out


def output(pos: np.ndarray, perm: np.ndarray, ext: np.ndarray) -> np.ndarray:
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    perm = np.ascontiguousarray(perm, dtype=np.int32)
    ext = np.ascontiguousarray(ext, dtype=np.float32)
    n = perm.shape[0]
    out = np.empty((3, n), np.float32)
    lib().orc_output(_p(pos), _p(perm), _p(ext), n, _p(out))
    return out


def bruteforce(pos: np.ndarray, k: int):
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    n = pos.shape[1]
    lists = np.empty((n, k), np.int32)
    d = np.empty((n, k), np.float32)
    lib().orc_bruteforce(_p(pos), n, k, _p(lists), _p(d))
    return lists, d


def select_check(xyz: np.ndarray, k: int):
    """Certification rule of the block-selection kNN against the ring search
    (brute force; small clouds): (certified rows, certified rows whose ring-search
    list is not the k nearest in order, certified rows with another stop level)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    st = np.zeros(3, np.int64)
    lib().orc_select_check(_p(xyz), xyz.shape[0], k, _p(st))
    return tuple(int(v) for v in st)


def knn_timed(xyz: np.ndarray, k: int, stride: int):
    """(t_build, t_query) seconds for the grid build plus every stride-th query."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    tb, tq = C.c_double(0), C.c_double(0)
    lib().orc_knn_timed(_p(xyz), xyz.shape[0], k, stride, C.byref(tb), C.byref(tq))
    return tb.value, tq.value


# ---------------------------------------------------------------------------
# Learned search proposal (extension of this project; no reference counterpart)

PROPOSAL_CLASSES = 16
PROPOSAL_BOXES = [(0, 1), (0, 2), (0, 3), (0, 4), (0, 5), (0, 6), (1, 4), (1, 5),
                  (1, 6), (2, 4), (2, 5), (2, 6), (3, 4), (3, 5), (3, 6)]


def proposal_data(xyz: np.ndarray, k: int):
    """Features [n,8] and labels [n] (sorted space) from the plain grid kNN."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    n = xyz.shape[0]
    feats = np.empty((n, 8), np.float32)
    labels = np.empty(n, np.uint8)
    lib().orc_proposal_data(_p(xyz), n, k, _p(feats), _p(labels))
    return feats, labels


def knn_proposal(xyz: np.ndarray, k: int, cls: np.ndarray):
    """Grid kNN driven by per-query proposal classes (sorted space).  The lists
    must equal knn()'s; `certified` marks queries answered by the box search."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    cls = np.ascontiguousarray(cls, dtype=np.uint8)
    n = xyz.shape[0]
    lists = np.empty((n, k), np.int32)
    cert = np.empty(n, np.uint8)
    level = np.empty(n, np.int32)
    bv, pv = C.c_longlong(0), C.c_longlong(0)
    inv = lib().orc_knn_proposal(_p(xyz), n, k, _p(cls), _p(lists), _p(cert), _p(level), C.byref(bv), C.byref(pv))
    return dict(lists=lists, certified=cert, level=level, invalid=inv, box_visited=bv.value,
                plain_visited=pv.value)


# Proposal network (MLP 8 -> 32 -> 32 -> 16, ReLU, softmax), restated in float64
# for checking the device kernels.  params: the binary16 parameter vector in
# the layout W1[32][8] b1 W2[32][32] b2 W3[16][32] b3.
def _mlp_unpack(params: np.ndarray):
    params = np.asarray(params)
    # binary16 parameter vectors are used at their binary16 values; float64
    # vectors (finite-difference checks) as given
    p = params.copy() if params.dtype == np.float64 else params.astype(np.float16).astype(np.float64)
    sizes = [("W1", (32, 8)), ("b1", (32,)), ("W2", (32, 32)), ("b2", (32,)), ("W3", (16, 32)), ("b3", (16,))]
    out, o = {}, 0
    for name, shp in sizes:
        m = int(np.prod(shp))
        out[name] = p[o:o + m].reshape(shp)
        o += m
    assert o == p.size == 1872
    return out


def mlp_forward(params: np.ndarray, feats: np.ndarray):
    """Returns (h1, h2, logits) for feats [m, 8]."""
    P = _mlp_unpack(params)
    x = np.asarray(feats, dtype=np.float64)
    h1 = np.maximum(x @ P["W1"].T + P["b1"], 0.0)
    h2 = np.maximum(h1 @ P["W2"].T + P["b2"], 0.0)
    return h1, h2, h2 @ P["W3"].T + P["b3"]


def mlp_loss_grad(params: np.ndarray, feats: np.ndarray, labels: np.ndarray):
    """Mean cross-entropy and its gradient w.r.t. the parameter vector (float64)."""
    P = _mlp_unpack(params)
    x = np.asarray(feats, dtype=np.float64)
    y = np.asarray(labels).astype(np.int64)
    m = x.shape[0]
    h1, h2, z = mlp_forward(params, x)
    z = z - z.max(1, keepdims=True)
    e = np.exp(z)
    s = e.sum(1, keepdims=True)
    loss = float(np.mean(np.log(s[:, 0]) - z[np.arange(m), y]))
    d3 = e / s
    d3[np.arange(m), y] -= 1.0
    d3 /= m
    d2 = (d3 @ P["W3"]) * (h2 > 0)
    d1 = (d2 @ P["W2"]) * (h1 > 0)
    g = np.concatenate([(d1.T @ x).ravel(), d1.sum(0), (d2.T @ h1).ravel(), d2.sum(0), (d3.T @ h2).ravel(),
                        d3.sum(0)])
    return loss, g


def mlp_classes(params: np.ndarray, feats: np.ndarray, tau: float) -> np.ndarray:
    """Smallest class whose cumulative softmax probability reaches tau."""
    _, _, z = mlp_forward(params, feats)
    e = np.exp(z - z.max(1, keepdims=True))
    cdf = np.cumsum(e, 1) / e.sum(1, keepdims=True)
    return np.minimum((cdf < tau).sum(1), 15).astype(np.uint8)
