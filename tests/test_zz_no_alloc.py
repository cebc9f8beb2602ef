"""egt_taubin_noalloc: Taubin smoothing for callers that cannot allocate device
memory -- a host whose own allocator owns all GPU memory, or a real-time loop
that cannot take cudaMalloc's device synchronisation.

The entry point is called through the C ABI on device buffers the test owns
and must reproduce the regular egt_taubin result of a provider handle bit for
bit (both accumulate every row in list order with the same arithmetic), and
stay within 1e-6 of the bounding-box diagonal of the FP64 oracle, on two calls
in a row (the shared scratch array keeps the first call's contents, which the
second call must not depend on).  The file is named so that pytest collects it
last; it needs nothing from the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from golden_util import bbox_diag
from multigpuegtsmoothing_b200 import datagen

pytestmark = pytest.mark.gpu


def test_taubin_noalloc_matches_handle_taubin(capi, oracle):
    import torch

    xyz = datagen.sphere_cloud(30000, 0.005, 41)
    iters, lam, mu = 12, 0.63, -0.64
    g = capi.GridStructure(xyz)
    g.GRIDCUDAKNNSELF_COMPACT(24)
    egt = capi.EGT_CUDA(g)
    egt.Filter(0.65)
    start = g.sorted_positions()                      # (3, n) before smoothing
    lists = g.sorted_lists()
    off_p, col_p, nnz = C.c_void_p(), C.c_void_p(), C.c_int64()
    capi._check(capi.lib().egt_get_csr(g.handle, C.byref(off_p), C.byref(col_p), C.byref(nnz)))
    n = start.shape[1]
    # inputs/outputs owned by the caller (device float4 x,y,z,w)
    pin = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    pin[:, :3] = torch.from_numpy(start.T.copy()).cuda()
    pout = torch.empty_like(pin)
    torch.cuda.synchronize()
    results = []
    for _ in range(2):
        pout.fill_(float("nan"))
        torch.cuda.synchronize()
        st = capi.lib().egt_taubin_noalloc(C.c_void_p(pin.data_ptr()), C.c_void_p(pout.data_ptr()), off_p,
                                           col_p, n, iters, lam, mu, None)
        assert st == 0, capi.lib().egt_last_error()
        torch.cuda.synchronize()
        results.append(pout[:, :3].cpu().numpy().T.copy())
    # the regular entry point on the provider handle
    egt.Taubin(iters, lam, mu)
    want = g.sorted_positions()
    scale = g.GetMaxExtent() - g.GetMinExtent()
    tol = 1e-6 * bbox_diag(xyz)
    p64 = oracle.taubin_f64(start, lists, iters, lam, mu)
    for got in results:
        assert np.array_equal(got, want)
        assert np.abs(got - p64).max() * scale <= tol
    assert np.array_equal(results[0], results[1])
    # zero iterations on aliased buffers: nothing to do, the positions stay
    st = capi.lib().egt_taubin_noalloc(C.c_void_p(pout.data_ptr()), C.c_void_p(pout.data_ptr()), off_p, col_p, n,
                                       0, lam, mu, None)
    assert st == 0, capi.lib().egt_last_error()
    torch.cuda.synchronize()
    assert np.array_equal(pout[:, :3].cpu().numpy().T, results[1])


def test_taubin_noalloc_rejects_oversize(capi):
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    st = capi.lib().egt_taubin_noalloc(dummy, dummy, dummy, dummy, (1 << 20) + 1, 1, 0.63, -0.64, None)
    assert st == -2
    assert b"capacity" in capi.lib().egt_last_error()
