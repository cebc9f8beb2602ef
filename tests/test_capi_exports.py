"""The C-ABI library loads and exports every entry point its header declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os

from multigpuegtsmoothing_b200 import capi


def test_library_exports_header_symbols():
    L = capi.lib()
    names = capi.exported_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_default_config():
    L = capi.lib()
    assert b"sm_100a" in L.egt_version()
    c = capi.default_config()
    assert c.bucket_count == 1024 and abs(c.eps - 1e-6) < 1e-12
    assert c.max_points_in_cell == 100000 and c.threshold == 1e8
    assert c.knn_mode == 3  # EGT_KNN_TILE


def test_null_arguments_rejected_without_gpu():
    L = capi.lib()
    h = ctypes.c_void_p()
    # argument checks happen before any CUDA call
    assert L.egt_create_cloud(None, 10, None, None, ctypes.byref(h)) == -2
    assert L.egt_knn(None, 10, None) == -2
    assert b"null" in L.egt_last_error()


def test_header_lists_reference_interfaces():
    hdr = open(os.path.join(os.path.dirname(capi.HERE), "include", "egt_b200.h")).read()
    for ref in ("GRIDCUDAKNNSELF_COMPACT", "GetNeighborsFromTriangles", "PerformSmoothing", "GetNormals",
                "getOutputPoints", "KNNInterface"):
        assert ref in hdr
