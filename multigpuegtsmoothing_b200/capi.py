"""Python mirror of the reference's provider/consumer interface over the C ABI.

The reference drives its path through C++ classes: a provider
(``GridStructure`` / ``GridMeshCuda``, both ``KNNInterface``), the smoother
``EGT_CUDA``, ``Normal_CUDA`` and ``getOutputPoints`` (reference main.cpp:106-121).
This module keeps those names and argument meanings over
``lib/libegt_b200.so`` (include/egt_b200.h) so that host code and tests read
like the reference's own call sequence:

    g = GridStructure(xyz)                    # GridStructure(mesh, 1, 1e-6, 1024, 4)
    g.GRIDCUDAKNNSELF_COMPACT(40, 1e8)
    EGT_CUDA(g).PerformSmoothing(150, 0.63, -0.64, 0.65)
    nx, ny, nz = Normal_CUDA(g).GetNormals()
    x, y, z = getOutputPoints(g)

There is no fallback: if the CUDA library is missing or no GPU is present the
calls raise.  Arrays cross the boundary as numpy arrays (host memory).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libegt_b200.so")

EGT_OK = 0
_ERR_NAMES = {-1: "EGT_ERR_CUDA", -2: "EGT_ERR_ARG", -3: "EGT_ERR_CAP_EXCEEDED", -4: "EGT_ERR_TIMEOUT",
              -5: "EGT_ERR_STATE", -6: "EGT_ERR_NOMEM"}


class EgtError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_ERR_NAMES.get(status, status)}: {msg}")
        self.status = status


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("eps", C.c_float), ("bucket_count", C.c_int), ("threshold", C.c_float),
                ("max_points_in_cell", C.c_int), ("knn_mode", C.c_int), ("warps_per_block", C.c_int),
                ("normals_gap_tol", C.c_float)]


class Views(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("lists", C.c_void_p),
                ("perm", C.c_void_p), ("normals", C.c_void_p), ("n", C.c_int64), ("k", C.c_int),
                ("min_extent", C.c_float), ("max_extent", C.c_float)]


class Timings(C.Structure):
    _fields_ = [("grid_ms", C.c_float), ("knn_ms", C.c_float), ("egt_ms", C.c_float), ("taubin_ms", C.c_float),
                ("normals_ms", C.c_float), ("orient_ms", C.c_float), ("output_ms", C.c_float),
                ("levels_used", C.c_int), ("invalid_queries", C.c_int64), ("csr_nnz", C.c_int64),
                ("normals_fp64", C.c_int64), ("msf_edges", C.c_int64), ("components", C.c_int),
                ("egt_kernel_ms", C.c_float), ("propose_ms", C.c_float), ("box_queries", C.c_int64),
                ("certified_queries", C.c_int64), ("exact_reruns", C.c_int64),
                ("knn_evaluations", C.c_int64), ("egt_tests", C.c_int64),
                ("taubin_tiles", C.c_int64), ("taubin_spill_tiles", C.c_int64), ("knn_fallback", C.c_int64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class BatchTimings(C.Structure):
    _fields_ = [("grid_ms", C.c_float), ("knn_ms", C.c_float), ("egt_ms", C.c_float), ("taubin_ms", C.c_float),
                ("output_ms", C.c_float), ("tune_ms", C.c_float), ("clouds", C.c_int), ("points", C.c_int64),
                ("invalid_queries", C.c_int64), ("exact_reruns", C.c_int64), ("csr_nnz", C.c_int64),
                ("knn_chunk", C.c_int), ("taubin_mode", C.c_int), ("fused", C.c_int), ("fused_ms", C.c_float),
                ("separate_ms", C.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


def lib() -> C.CDLL:
    """Loads lib/libegt_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `make -C multigpuegtsmoothing_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, f32 = C.c_void_p, C.c_int, C.c_int64, C.c_float
        hp = C.POINTER(C.c_void_p)
        sigs = {
            "egt_default_config": (None, [C.POINTER(Config)]),
            "egt_last_error": (C.c_char_p, []),
            "egt_version": (C.c_char_p, []),
            "egt_create_cloud": (i32, [vp, i64, C.POINTER(Config), vp, hp]),
            "egt_create_cloud_device": (i32, [vp, i64, C.POINTER(Config), vp, hp]),
            "egt_create_mesh": (i32, [vp, i64, vp, i64, C.POINTER(Config), vp, hp]),
            "egt_knn": (i32, [vp, i32, vp]),
            "egt_knn_host": (i32, [vp, i32, vp, vp]),
            "egt_knn_query": (i32, [vp, vp, i64, i32, vp, C.POINTER(C.c_int64), vp]),
            "egt_orient_kruskal": (i32, [vp, vp, vp, vp, vp, vp, vp, i32, i32, i32, i32, vp]),
            "egt_mesh_1ring": (i32, [vp, i32, vp]),
            "egt_smooth": (i32, [vp, i32, f32, f32, f32, vp]),
            "egt_filter": (i32, [vp, f32, vp]),
            "egt_taubin": (i32, [vp, i32, f32, f32, vp]),
            "egt_normals": (i32, [vp, vp, vp, vp, vp]),
            "egt_output": (i32, [vp, vp, vp, vp, vp]),
            "egt_output_device": (i32, [vp, vp, vp, vp, vp]),
            "egt_get_knn_host": (i32, [vp, vp, vp]),
            "egt_get_views": (i32, [vp, C.POINTER(Views)]),
            "egt_commit_views": (i32, [vp, vp, vp, vp, vp]),
            "egt_free_device": (i32, [vp]),
            "egt_set_threshold": (i32, [vp, f32, vp]),
            "egt_get_timings": (i32, [vp, C.POINTER(Timings)]),
            "egt_get_csr": (i32, [vp, hp, hp, C.POINTER(C.c_int64)]),
            "egt_copy_to_host": (i32, [vp, vp, vp, i64]),
            "egt_update_points_device": (i32, [vp, vp, vp]),
            "egt_kernel_launches": (i64, []),
            "egt_taubin_noalloc": (i32, [vp, vp, vp, vp, i64, i32, f32, f32, vp]),
            "egt_taubin_halfstep": (i32, [vp, vp, vp, vp, i64, f32, i32, vp]),
            "egt_destroy": (None, [vp]),
            "egt_proposal_create": (i32, [i32, i32, C.c_uint64, hp]),
            "egt_proposal_destroy": (None, [vp]),
            "egt_proposal_collect": (i32, [vp, vp, i32]),
            "egt_proposal_samples": (i64, [vp]),
            "egt_proposal_train": (i32, [vp, i32, i32, f32, vp]),
            "egt_proposal_gradients": (i32, [vp, vp, vp, i32, vp, vp]),
            "egt_proposal_get_params": (i32, [vp, vp]),
            "egt_proposal_set_params": (i32, [vp, vp]),
            "egt_proposal_set_tau": (i32, [vp, f32]),
            "egt_proposal_get_tau": (f32, [vp]),
            "egt_proposal_tune": (i32, [vp, vp, vp, i32, vp]),
            "egt_proposal_inspect": (i32, [vp, vp, vp, vp, vp]),
            "egt_knn_learned": (i32, [vp, i32, vp, vp]),
            "egt_attach_proposal": (i32, [vp, vp]),
            "egt_batch_create": (i32, [vp, vp, vp, i32, C.POINTER(Config), vp, hp]),
            "egt_batch_knn": (i32, [vp, vp]),
            "egt_batch_filter": (i32, [vp, f32, vp]),
            "egt_batch_taubin": (i32, [vp, i32, f32, f32, vp]),
            "egt_batch_run": (i32, [vp, i32, f32, f32, f32, vp]),
            "egt_batch_set_tuning": (i32, [vp, i32, i32]),
            "egt_batch_output": (i32, [vp, vp, vp]),
            "egt_batch_get_knn_host": (i32, [vp, i32, vp]),
            "egt_batch_get_timings": (i32, [vp, C.POINTER(BatchTimings)]),
            "egt_batch_destroy": (None, [vp]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    """Names of every entry point declared in include/egt_b200.h."""
    import re
    hdr = os.path.join(os.path.dirname(HERE), "include", "egt_b200.h")
    txt = open(hdr).read()
    return sorted(set(re.findall(r"^\s*(?:egt_status|void|int64_t|int|float|const char\*)\s+(egt_\w+)\s*\(", txt, re.M)))


def _check(st: int):
    if st != EGT_OK:
        raise EgtError(st, lib().egt_last_error().decode())


def default_config(**kw) -> Config:
    c = Config()
    lib().egt_default_config(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class _Handle:
    """Owns one egt_handle (the provider's device state)."""

    def __init__(self, h: C.c_void_p, stream: int = 0):
        self._h = h
        self.stream = C.c_void_p(stream) if stream else None

    @property
    def handle(self):
        if self._h is None:
            raise EgtError(-5, "handle destroyed")
        return self._h

    def close(self):
        if self._h is not None:
            lib().egt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- KNNInterface getters (KNNInterface.cuh:8-31) ---------------------------------
    def views(self) -> Views:
        v = Views()
        _check(lib().egt_get_views(self.handle, C.byref(v)))
        return v

    def pointsRefCount(self) -> int:
        return int(self.views().n)

    def NeighborCount(self) -> int:
        return int(self.views().k)

    def GetMinExtent(self) -> float:
        return float(self.views().min_extent)

    def GetMaxExtent(self) -> float:
        return float(self.views().max_extent)

    def GetNumberOfCards(self) -> int:
        return 1

    def isReady(self) -> bool:
        return bool(self.views().lists)

    def _d2h(self, ptr, shape, dtype):
        out = np.empty(shape, dtype=dtype)
        if out.nbytes:
            _check(lib().egt_copy_to_host(self.handle, _ptr(out), C.c_void_p(ptr), out.nbytes))
        return out

    def sorted_positions(self) -> np.ndarray:
        """(3, n) float32: GetRefPointsX/Y/Z()[0] (sorted, normalised)."""
        v = self.views()
        n = int(v.n)
        return np.stack([self._d2h(v.x, n, np.float32), self._d2h(v.y, n, np.float32),
                         self._d2h(v.z, n, np.float32)])

    def sorted_lists(self) -> np.ndarray:
        """(n, k) int32: GetKNNIndexesInPartitions()[0] (sorted space, -1 padded)."""
        v = self.views()
        return self._d2h(v.lists, (int(v.n), int(v.k)), np.int32)

    def GetOriginalRefIndexes(self) -> np.ndarray:
        v = self.views()
        return self._d2h(v.perm, int(v.n), np.int32)

    def sorted_normals(self) -> Optional[np.ndarray]:
        v = self.views()
        if not v.normals:
            return None
        return self._d2h(v.normals, (3, int(v.n)), np.float32)

    def GetKNNIndexes(self) -> np.ndarray:
        """(n, k) int32 in original ids and original row order (GridKNNCuda.cu:1941-1968)."""
        v = self.views()
        out = np.empty((int(v.n), int(v.k)), np.int32)
        _check(lib().egt_get_knn_host(self.handle, _ptr(out), self.stream))
        return out

    def csr(self) -> Tuple[np.ndarray, np.ndarray]:
        off = C.c_void_p()
        col = C.c_void_p()
        nnz = C.c_int64()
        _check(lib().egt_get_csr(self.handle, C.byref(off), C.byref(col), C.byref(nnz)))
        n = self.pointsRefCount()
        return self._d2h(off.value, n + 1, np.int32), self._d2h(col.value, int(nnz.value), np.int32)

    def timings(self) -> dict:
        t = Timings()
        _check(lib().egt_get_timings(self.handle, C.byref(t)))
        return t.as_dict()


class GridStructure(_Handle):
    """Point-cloud provider: GridStructure(mesh, 1, eps, 1024, 4) (GridKNNCuda.cu:1165-1205)."""

    def __init__(self, xyz: np.ndarray, num_cards: int = 1, eps: float = 1e-6, bucketCount: int = 1024,
                 maxDivision: int = 4, config: Optional[Config] = None, stream: int = 0, device_ptr: int = 0,
                 n: int = 0):
        if num_cards != 1:
            raise EgtError(-2, "this build runs on one GPU (num_cards must be 1)")
        cfg = config or default_config()
        cfg.eps = eps
        cfg.bucket_count = bucketCount
        h = C.c_void_p()
        s = C.c_void_p(stream) if stream else None
        if device_ptr:
            _check(lib().egt_create_cloud_device(C.c_void_p(device_ptr), n, C.byref(cfg), s, C.byref(h)))
        else:
            xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
            _check(lib().egt_create_cloud(_ptr(xyz), xyz.shape[0], C.byref(cfg), s, C.byref(h)))
        super().__init__(h, stream)

    def UpdatePointsDevice(self, device_ptr: int):
        """Rebuild normalisation, cell sort and hierarchy for new device positions (same n)."""
        _check(lib().egt_update_points_device(self.handle, C.c_void_p(device_ptr), self.stream))

    def GRIDCUDAKNNSELF_COMPACT(self, k: int, thres: Optional[float] = None):
        """GRIDCUDAKNNSELF_COMPACT(k, thres): thres (the reference's units) is set
        on the handle when given; otherwise the handle's threshold stays."""
        if thres is not None:
            _check(lib().egt_set_threshold(self.handle, float(thres), self.stream))
        _check(lib().egt_knn(self.handle, int(k), self.stream))

    def knn_host(self, k: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        """GRIDCUDAKNNSELF_COMPACT(k) then GetKNNIndexes() in one call, with the
        host copy overlapped with the search (egt_knn_host).  out: optional
        (n, k) int32 C-contiguous host array (pinned memory overlaps best)."""
        n = self.pointsRefCount()
        if out is None:
            out = np.empty((n, int(k)), np.int32)
        if out.dtype != np.int32 or out.shape != (n, int(k)) or not out.flags["C_CONTIGUOUS"]:
            raise EgtError(-2, "knn_host: out must be a C-contiguous (n, k) int32 array")
        _check(lib().egt_knn_host(self.handle, int(k), _ptr(out), self.stream))
        return out

    def GRIDCUDAKNNCompact(self, queries: np.ndarray, k: int) -> Tuple[np.ndarray, int]:
        """Query-vs-reference kNN (GridKNNCuda.cu:1645-1968) against this
        provider's points: (nq, k) int32 original reference ids in query order
        (GetKNNIndexes layout) and the number of invalid queries."""
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, 3)
        out = np.empty((q.shape[0], int(k)), np.int32)
        inv = C.c_int64(0)
        _check(lib().egt_knn_query(self.handle, _ptr(q), q.shape[0], int(k), _ptr(out), C.byref(inv), self.stream))
        return out, int(inv.value)

    def GRIDCUDAKNNSELF_LEARNED(self, k: int, proposal: "SearchProposal"):
        """The same search driven by a learned proposal: lists bit-identical to
        GRIDCUDAKNNSELF_COMPACT (no reference counterpart)."""
        _check(lib().egt_knn_learned(self.handle, int(k), proposal.handle, self.stream))


class GridMeshCuda(_Handle):
    """Mesh provider: GridMeshCuda(mesh, 1, eps, 1024) (GridMeshCuda1.cu:247-414)."""

    def __init__(self, xyz: np.ndarray, tris: np.ndarray, num_cards: int = 1, eps: float = 1e-6,
                 bucketCount: int = 1024, config: Optional[Config] = None, stream: int = 0):
        if num_cards != 1:
            raise EgtError(-2, "this build runs on one GPU (num_cards must be 1)")
        cfg = config or default_config()
        cfg.eps = eps
        cfg.bucket_count = bucketCount
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        tris = np.ascontiguousarray(tris, dtype=np.uint32).reshape(-1, 3)
        h = C.c_void_p()
        s = C.c_void_p(stream) if stream else None
        _check(lib().egt_create_mesh(_ptr(xyz), xyz.shape[0], _ptr(tris), tris.shape[0], C.byref(cfg), s,
                                     C.byref(h)))
        super().__init__(h, stream)

    def GetNeighborsFromTriangles(self, k: int):
        _check(lib().egt_mesh_1ring(self.handle, int(k), self.stream))


class EGT_CUDA:
    """EGT_CUDA(provider).PerformSmoothing(iters, lambda, mu, alpha) (EGT_CUDA.cu:392-648)."""

    def __init__(self, provider: _Handle):
        self.p = provider

    def PerformSmoothing(self, iterationCount: int, lambda_: float = 0.63, mu: float = -0.64,
                         alpha: float = 1e-8):
        _check(lib().egt_smooth(self.p.handle, int(iterationCount), lambda_, mu, alpha, self.p.stream))

    def Filter(self, alpha: float):
        _check(lib().egt_filter(self.p.handle, alpha, self.p.stream))

    def Taubin(self, iterationCount: int, lambda_: float = 0.63, mu: float = -0.64):
        _check(lib().egt_taubin(self.p.handle, int(iterationCount), lambda_, mu, self.p.stream))


class Normal_CUDA:
    """Normal_CUDA(provider).GetNormals() (Normal_CUDA.cu:304-788): oriented normals, original order."""

    def __init__(self, provider: _Handle):
        self.p = provider

    def GetNormals(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        n = self.p.pointsRefCount()
        nx, ny, nz = (np.empty(n, np.float32) for _ in range(3))
        _check(lib().egt_normals(self.p.handle, _ptr(nx), _ptr(ny), _ptr(nz), self.p.stream))
        return nx, ny, nz


def kernel_launches() -> int:
    """Kernels launched by the library from this host thread so far."""
    return int(lib().egt_kernel_launches())


def getOutputPoints(provider: _Handle) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Denormalised positions in original order (getOutputPoints.cu:34-63)."""
    n = provider.pointsRefCount()
    x, y, z = (np.empty(n, np.float32) for _ in range(3))
    _check(lib().egt_output(provider.handle, _ptr(x), _ptr(y), _ptr(z), provider.stream))
    return x, y, z


def orient_kruskal(knn: np.ndarray, nx: np.ndarray, ny: np.ndarray, nz: np.ndarray, x=None, y=None, z=None,
                   N: Optional[int] = None, k: Optional[int] = None, k_use: Optional[int] = None,
                   device: int = 0) -> None:
    """orient_kruskal(knn, nx, ny, nz, x, y, z, N, k, k_use) (MST.cpp:399-423):
    the reference's CPU normal orienter, computed on the GPU.  knn: (N, k)
    int32 (or flat N*k); nx, ny, nz: float32 arrays of N, oriented in place
    (they must be contiguous float32).  x, y, z are not read."""
    knn = np.ascontiguousarray(knn, dtype=np.int32)
    for a in (nx, ny, nz):
        if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous):
            raise TypeError("orient_kruskal: nx, ny, nz must be contiguous float32 arrays (oriented in place)")
    n = int(N) if N is not None else nx.shape[0]
    kk = int(k) if k is not None else (knn.shape[1] if knn.ndim == 2 else knn.size // max(n, 1))
    ku = int(k_use) if k_use is not None else kk
    if knn.size < n * kk or min(nx.size, ny.size, nz.size) < n:
        raise ValueError("orient_kruskal: arrays smaller than N*k / N")
    _check(lib().egt_orient_kruskal(_ptr(knn), _ptr(nx), _ptr(ny), _ptr(nz), None, None, None, n, kk, ku,
                                    int(device), None))


PROPOSAL_PARAMS = 1872
PROPOSAL_CLASSES = 16
PROPOSAL_FEATURES = 8


class SearchProposal:
    """Learned search proposal (egt_proposal_*; no reference counterpart).

    An MLP 8 -> 32 -> 32 -> 16 with binary16 parameters proposes, per query, a
    box of grid cells for the kNN search; the search certifies the box result
    or falls back to the plain search, so lists never change.  Training data
    comes from providers that ran the plain search (collect), training runs on
    the GPU (train), and tune() picks the class threshold by timing.
    """

    def __init__(self, k: int, seed: int = 0, device: int = 0):
        h = C.c_void_p()
        _check(lib().egt_proposal_create(int(device), int(k), C.c_uint64(seed), C.byref(h)))
        self._h = h
        self.k = int(k)

    @property
    def handle(self):
        if self._h is None:
            raise EgtError(-5, "proposal destroyed")
        return self._h

    def close(self):
        if self._h is not None:
            lib().egt_proposal_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def collect(self, provider: _Handle, stride: int = 1):
        _check(lib().egt_proposal_collect(self.handle, provider.handle, int(stride)))

    @property
    def samples(self) -> int:
        return int(lib().egt_proposal_samples(self.handle))

    def train(self, steps: int, batch: int = 4096, lr: float = 3e-3) -> np.ndarray:
        loss = np.zeros(max(int(steps), 1), np.float32)
        _check(lib().egt_proposal_train(self.handle, int(steps), int(batch), float(lr), _ptr(loss)))
        return loss[:int(steps)]

    def gradients(self, feats: np.ndarray, labels: np.ndarray) -> Tuple[np.ndarray, float]:
        feats = np.ascontiguousarray(feats, dtype=np.float32).reshape(-1, PROPOSAL_FEATURES)
        labels = np.ascontiguousarray(labels, dtype=np.uint8).reshape(-1)
        g = np.zeros(PROPOSAL_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        _check(lib().egt_proposal_gradients(self.handle, _ptr(feats), _ptr(labels), feats.shape[0], _ptr(g),
                                            _ptr(loss)))
        return g, float(loss[0])

    def params(self) -> np.ndarray:
        """binary16 parameters (np.float16, layout W1[32][8] b1 W2[32][32] b2 W3[16][32] b3)."""
        out = np.zeros(PROPOSAL_PARAMS, np.float16)
        _check(lib().egt_proposal_get_params(self.handle, _ptr(out)))
        return out

    def set_params(self, params: np.ndarray):
        params = np.ascontiguousarray(params, dtype=np.float16)
        _check(lib().egt_proposal_set_params(self.handle, _ptr(params)))

    @property
    def tau(self) -> float:
        return float(lib().egt_proposal_get_tau(self.handle))

    @tau.setter
    def tau(self, v: float):
        _check(lib().egt_proposal_set_tau(self.handle, float(v)))

    def tune(self, provider: _Handle, taus=(0.6, 0.75, 0.85, 0.92, 0.97)) -> dict:
        t = np.ascontiguousarray(taus, dtype=np.float32)
        ms = np.zeros(len(t), np.float32)
        _check(lib().egt_proposal_tune(self.handle, provider.handle, _ptr(t), len(t), _ptr(ms)))
        return dict(zip([float(x) for x in t], [float(x) for x in ms]))

    def inspect(self, provider: _Handle, feats=True, labels=True, classes=True):
        n = provider.pointsRefCount()
        f = np.zeros((n, PROPOSAL_FEATURES), np.float32) if feats else None
        l = np.zeros(n, np.uint8) if labels else None
        c = np.zeros(n, np.uint8) if classes else None
        _check(lib().egt_proposal_inspect(self.handle, provider.handle, None if f is None else _ptr(f),
                                          None if l is None else _ptr(l), None if c is None else _ptr(c)))
        return f, l, c


class Batch:
    """Many independent clouds through kNN -> EGT -> Taubin with one launch per
    stage (egt_batch_*; no reference counterpart).  Each cloud's results equal
    those of its own GridStructure run through the same calls."""

    def __init__(self, clouds, config: Optional[Config] = None, stream: int = 0):
        xyzs = [np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3) for x, _ in clouds]
        ks = np.ascontiguousarray([int(k) for _, k in clouds], dtype=np.int32)
        self.offsets = np.zeros(len(xyzs) + 1, np.int64)
        self.offsets[1:] = np.cumsum([x.shape[0] for x in xyzs])
        self.k = ks
        allx = np.ascontiguousarray(np.concatenate(xyzs), dtype=np.float32)
        cfg = config or default_config()
        h = C.c_void_p()
        self.stream = C.c_void_p(stream) if stream else None
        _check(lib().egt_batch_create(_ptr(allx), _ptr(self.offsets), _ptr(ks), len(xyzs), C.byref(cfg), self.stream,
                                      C.byref(h)))
        self._h = h

    @property
    def handle(self):
        if self._h is None:
            raise EgtError(-5, "batch destroyed")
        return self._h

    def close(self):
        if self._h is not None:
            lib().egt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def knn(self):
        _check(lib().egt_batch_knn(self.handle, self.stream))

    def filter(self, alpha: float):
        _check(lib().egt_batch_filter(self.handle, float(alpha), self.stream))

    def taubin(self, iters: int, lambda_: float = 0.63, mu: float = -0.64):
        _check(lib().egt_batch_taubin(self.handle, int(iters), float(lambda_), float(mu), self.stream))

    def run(self, iters: int = 150, lambda_: float = 0.63, mu: float = -0.64, alpha: float = 0.65):
        _check(lib().egt_batch_run(self.handle, int(iters), float(lambda_), float(mu), float(alpha), self.stream))

    def set_tuning(self, knn_chunk: int, taubin_mode: int):
        _check(lib().egt_batch_set_tuning(self.handle, int(knn_chunk), int(taubin_mode)))

    def output(self):
        """List of per-cloud (n_c, 3) float32 positions in original order."""
        out = np.empty((int(self.offsets[-1]), 3), np.float32)
        _check(lib().egt_batch_output(self.handle, _ptr(out), self.stream))
        return [out[self.offsets[c]:self.offsets[c + 1]] for c in range(len(self.k))]

    def knn_host(self, cloud: int) -> np.ndarray:
        n = int(self.offsets[cloud + 1] - self.offsets[cloud])
        out = np.empty((n, int(self.k[cloud])), np.int32)
        _check(lib().egt_batch_get_knn_host(self.handle, int(cloud), _ptr(out)))
        return out

    def timings(self) -> dict:
        t = BatchTimings()
        _check(lib().egt_batch_get_timings(self.handle, C.byref(t)))
        return t.as_dict()
