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
        L.orc_knn.argtypes = [vp, i32, i32, vp, vp, vp, vp, vp, vp, vp]
        L.orc_mesh_1ring.argtypes = [vp, i32, vp, i32, i32, vp, vp, vp, vp]
        L.orc_egt.argtypes = [vp, i32, i32, vp, f32, vp]
        L.orc_taubin_f32.argtypes = [vp, i32, i32, vp, i32, f32, f32]
        L.orc_taubin_f64.argtypes = [vp, i32, i32, vp, i32, C.c_double, C.c_double]
        L.orc_normals.argtypes = [vp, i32, i32, vp, i32, vp]
        L.orc_orient.restype = i32
        L.orc_orient.argtypes = [i32, i32, vp, vp, vp]
        L.orc_output.argtypes = [vp, vp, vp, i32, vp]
        L.orc_bruteforce.argtypes = [vp, i32, i32, vp, vp]
        L.orc_knn_timed.argtypes = [vp, i32, i32, i32, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def num_threads() -> int:
    return lib().orc_num_threads()


def knn(xyz: np.ndarray, k: int):
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
    inv = lib().orc_knn(_p(xyz), n, k, _p(lists), _p(pos), _p(perm), _p(ext), _p(level), _p(kth),
                        C.byref(visited))
    return dict(lists=lists, pos=pos, perm=perm, ext=ext, level=level, kth=kth, invalid=inv,
                visited=visited.value)


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


def orient(nrm: np.ndarray, lists: np.ndarray):
    """Orient sorted-space normals in place order; returns (normals, parent, ncomp)."""
    lists = np.ascontiguousarray(lists, dtype=np.int32)
    n, k = lists.shape
    out = np.array(nrm, dtype=np.float32, order="C", copy=True)
    parent = np.empty(n, np.int32)
    nc = lib().orc_orient(n, k, _p(lists), _p(out), _p(parent))
    return out, parent, nc


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


def knn_timed(xyz: np.ndarray, k: int, stride: int):
    """(t_build, t_query) seconds for the grid build plus every stride-th query."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    tb, tq = C.c_double(0), C.c_double(0)
    lib().orc_knn_timed(_p(xyz), xyz.shape[0], k, stride, C.byref(tb), C.byref(tq))
    return tb.value, tq.value
