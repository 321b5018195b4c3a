"""The allocation-free CRS SpMV entry point (smax_spmv_crs_noalloc).

It exists for callers that cannot call cudaMalloc: an application whose memory
pool already owns the GPU, a plugin whose host forbids device allocations, or a
loop that must not enter the allocator.  These tests call it through the C ABI
on device arrays and check its output against the regular entry point
(smax_kernel_run through the Interface mirror), within the tolerance the other
SpMV parity tests use, on two calls in a row (the shared scratch keeps the
previous call's contents, so the second call checks that nothing stale leaks).

This file is collected last (test_zz_*), so a run that stops at the first
failure has already run every other test; it also passes on its own.
"""
import ctypes

import numpy as np
import pytest

from helpers import gpu_spmv, normwise, rand_crs, tol

pytestmark = pytest.mark.gpu


def _noalloc(float_type, n_rows, n_cols, rp_d, col_d, val_d, x_d, y_d):
    from smaxkernels_b200 import _lib
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    rc = _lib.lib.smax_spmv_crs_noalloc(
        float_type, n_rows, n_cols, int(col_d.numel()), ctypes.c_void_p(rp_d.data_ptr()),
        ctypes.c_void_p(col_d.data_ptr()), ctypes.c_void_p(val_d.data_ptr()), ctypes.c_void_p(x_d.data_ptr()),
        ctypes.c_void_p(y_d.data_ptr()), ctypes.c_void_p(stream))
    return rc


@pytest.mark.parametrize("vt", [np.float64, np.float32])
def test_noalloc_matches_regular_entry_point_twice(vt):
    import torch
    from smaxkernels_b200 import _lib
    ft = 1 if vt == np.float64 else 0
    tdt = torch.float64 if vt == np.float64 else torch.float32
    # ragged rows, empty rows and a few long rows; n_cols != n_rows
    rp, col, val = rand_crs(30011, 60, 21, vt=vt, n_cols=40009, empty_frac=0.2, long_rows=(3000, 9000))
    n, n_cols = len(rp) - 1, 40009
    rng = np.random.default_rng(22)
    rp_d = torch.from_numpy(rp).cuda()
    col_d = torch.from_numpy(col).cuda()
    val_d = torch.from_numpy(val).cuda()
    for call in range(2):
        x = rng.uniform(-1, 1, n_cols).astype(vt)
        y_regular = gpu_spmv(rp, col, val, x)
        x_d = torch.from_numpy(x).cuda()
        y_d = torch.full((n,), float("nan"), dtype=tdt, device="cuda")
        torch.cuda.synchronize()
        assert _noalloc(ft, n, n_cols, rp_d, col_d, val_d, x_d, y_d) == _lib.OK, _lib.lib.smax_last_error()
        y = y_d.cpu().numpy()
        assert np.all(np.isfinite(y)), f"call {call}: rows left unwritten"
        assert normwise(y, y_regular) <= tol(vt), f"call {call}"


def test_noalloc_rejects_sizes_beyond_the_limit():
    from smaxkernels_b200 import _lib
    big = (1 << 24) + 1  # SMAX_NOALLOC_MAX_NNZ + 1
    rc = _lib.lib.smax_spmv_crs_noalloc(1, 1000, 1000, big, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                        ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert rc == _lib.ERR_BAD_ARG
    assert b"nnz" in _lib.lib.smax_last_error()
    rc = _lib.lib.smax_spmv_crs_noalloc(1, (1 << 20) + 1, 1000, 10, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                        ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert rc == _lib.ERR_BAD_ARG


def test_noalloc_reports_malformed_matrix():
    import torch
    from smaxkernels_b200 import _lib
    rp, col, val = rand_crs(500, 10, 23)
    col = col.copy()
    col[7] = 500  # out of range: rejected by the validation pass, never gathered
    rp_d, col_d, val_d = (torch.from_numpy(a).cuda() for a in (rp, col, val))
    x_d = torch.ones(500, dtype=torch.float64, device="cuda")
    y_d = torch.zeros(500, dtype=torch.float64, device="cuda")
    assert _noalloc(1, 500, 500, rp_d, col_d, val_d, x_d, y_d) == _lib.ERR_COL_OOB
