"""The allocation-free CRS SpMV entry point (smax_spmv_crs_noalloc).

It exists for callers that cannot call cudaMalloc: an application whose memory
pool already owns the GPU, a plugin whose host forbids device allocations, or a
loop that must not enter the allocator.  These tests call it through the C ABI
on device arrays and check its output against the regular entry point
(smax_kernel_run through the Interface mirror) and against the oracle, within
the tolerance the other SpMV parity tests use, on two calls in a row.  The
shared scratch keeps the previous call's contents, so the second call uses a
different, smaller matrix (fewer rows, more empty rows, another row layout):
any stale row-end bit, row list entry or slice rank from the first call would
show up in its result.

This file is collected last (test_zz_*), so a run that stops at the first
failure has already run every other test; it also passes on its own.
"""
import ctypes

import numpy as np
import pytest

from helpers import gpu_spmv, normwise, rand_crs, tol

pytestmark = pytest.mark.gpu

MAX_ROWS = 1 << 20  # SMAX_NOALLOC_MAX_ROWS
MAX_NNZ = 1 << 24   # SMAX_NOALLOC_MAX_NNZ


def _noalloc(float_type, n_rows, n_cols, rp_d, col_d, val_d, x_d, y_d, nnz=None):
    from smaxkernels_b200 import _lib
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    rc = _lib.lib.smax_spmv_crs_noalloc(
        float_type, n_rows, n_cols, int(col_d.numel()) if nnz is None else nnz, ctypes.c_void_p(rp_d.data_ptr()),
        ctypes.c_void_p(col_d.data_ptr()), ctypes.c_void_p(val_d.data_ptr()), ctypes.c_void_p(x_d.data_ptr()),
        ctypes.c_void_p(y_d.data_ptr()), ctypes.c_void_p(stream))
    return rc


def _run_noalloc(rp, col, val, x, n_cols):
    """y from the allocation-free entry point, y pre-filled with NaN so rows it
    leaves unwritten show."""
    import torch
    from smaxkernels_b200 import _lib
    ft = 1 if val.dtype == np.float64 else 0
    tdt = torch.float64 if val.dtype == np.float64 else torch.float32
    n = len(rp) - 1
    rp_d, col_d, val_d, x_d = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (rp, col, val, x))
    y_d = torch.full((n,), float("nan"), dtype=tdt, device="cuda")
    torch.cuda.synchronize()
    rc = _noalloc(ft, n, n_cols, rp_d, col_d, val_d, x_d, y_d)
    assert rc == _lib.OK, _lib.lib.smax_last_error()
    return y_d.cpu().numpy()


def _oracle_y(rp, col, val, x):
    from oracle.oracle import Oracle
    return Oracle().spmv_crs(rp, col, val, x)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
def test_noalloc_matches_regular_entry_point_and_oracle_twice(vt):
    rng = np.random.default_rng(22)
    cases = [
        # call 1: ragged rows, 20 % empty, a few long rows (carries across slices); n_cols != n_rows
        (rand_crs(30011, 60, 21, vt=vt, n_cols=40009, empty_frac=0.2, long_rows=(3000, 9000)), 40009),
        # call 2, right after: fewer rows, 60 % empty, other long-row positions, more columns than rows
        (rand_crs(7013, 25, 24, vt=vt, n_cols=9001, empty_frac=0.6, long_rows=(1500,)), 9001),
    ]
    for call, ((rp, col, val), n_cols) in enumerate(cases):
        x = rng.uniform(-1, 1, n_cols).astype(vt)
        y = _run_noalloc(rp, col, val, x, n_cols)
        assert np.all(np.isfinite(y)), f"call {call}: rows left unwritten"
        y_regular = gpu_spmv(rp, col, val, x, n_cols=n_cols)
        assert normwise(y, y_regular) <= tol(vt), f"call {call}: differs from the regular entry point"
        y_oracle = _oracle_y(rp, col, val, x.astype(np.float64) if vt == np.float64 else x)
        assert normwise(y, y_oracle) <= tol(vt), f"call {call}: differs from the oracle"
        if vt == np.float32:
            y64 = _oracle_y(rp, col, val.astype(np.float64), x.astype(np.float64))
            assert normwise(y, y64) <= tol(vt), f"call {call}: FP32 result against the FP64 oracle"


def _limit_matrix(seed=25):
    """n_rows = 2^20 and nnz = 2^24 exactly: ragged row lengths 0..32 (about
    3 % empty) trimmed to sum to 2^24, uniform random columns."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 33, MAX_ROWS).astype(np.int64)
    diff = int(lens.sum()) - MAX_NNZ
    step = 1 if diff > 0 else -1
    idx = rng.permutation(MAX_ROWS)
    k = 0
    while diff != 0:  # move lengths one at a time, keeping each in [0, 32]
        r = idx[k % MAX_ROWS]
        if (step > 0 and lens[r] > 0) or (step < 0 and lens[r] < 32):
            lens[r] -= step
            diff -= step
        k += 1
    rp = np.zeros(MAX_ROWS + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    col = rng.integers(0, MAX_ROWS, MAX_NNZ).astype(np.int32)
    val = rng.uniform(-1, 1, MAX_NNZ)
    return rp, col, val


def test_noalloc_at_the_size_limits():
    rp, col, val = _limit_matrix()
    assert len(rp) - 1 == MAX_ROWS and len(col) == MAX_NNZ
    x = np.random.default_rng(26).uniform(-1, 1, MAX_ROWS)
    y = _run_noalloc(rp, col, val, x, MAX_ROWS)
    assert np.all(np.isfinite(y))
    assert normwise(y, _oracle_y(rp, col, val, x)) <= 1e-12
    assert normwise(y, gpu_spmv(rp, col, val, x)) <= 1e-12


def test_noalloc_rejects_sizes_beyond_the_limit():
    from smaxkernels_b200 import _lib
    big = MAX_NNZ + 1
    rc = _lib.lib.smax_spmv_crs_noalloc(1, 1000, 1000, big, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                        ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert rc == _lib.ERR_BAD_ARG
    assert b"nnz" in _lib.lib.smax_last_error()
    rc = _lib.lib.smax_spmv_crs_noalloc(1, MAX_ROWS + 1, 1000, 10, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                        ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert rc == _lib.ERR_BAD_ARG


def _malformed_cases():
    """(name, row_ptr, col, expected status attribute).  Every bad value stays
    near the valid range: no case can make an access leave the caller's
    arrays or the scratch array, whatever the validation does."""
    rp, col, _ = rand_crs(500, 10, 23)
    nnz = len(col)
    out = []
    c = col.copy()
    c[7] = 500  # column out of range: rejected by the validation pass, never gathered
    out.append(("col_out_of_range", rp, c, "ERR_COL_OOB"))
    r = rp.copy()
    r[0] = 1  # row_ptr[0] != 0
    out.append(("row_ptr_0_not_zero", r, col, "ERR_BAD_ARG"))
    r = rp.copy()
    r[-1] = nnz - 1  # row_ptr[n] != nnz (the last row loses an entry)
    out.append(("row_ptr_n_not_nnz", r, col, "ERR_BAD_ARG"))
    r = rp.copy()
    k = int(np.argmax(np.diff(rp[1:-1]) > 0)) + 1  # an interior pair with rp[k] < rp[k+1]
    r[k], r[k + 1] = rp[k + 1], rp[k]  # decreasing row_ptr
    out.append(("row_ptr_decreasing", r, col, "ERR_BAD_ARG"))
    r = rp.copy()
    r[1] = -1  # negative entry: row_ptr = [0, -1, ...]
    out.append(("row_ptr_negative", r, col, "ERR_BAD_ARG"))
    return out


@pytest.mark.parametrize("case", _malformed_cases(), ids=lambda c: c[0])
def test_noalloc_reports_malformed_matrix(case):
    import torch
    from smaxkernels_b200 import _lib
    name, rp, col, status = case
    rng = np.random.default_rng(27)
    val = rng.uniform(-1, 1, len(col))
    rp_d, col_d, val_d = (torch.from_numpy(a).cuda() for a in (rp, col, val))
    x_d = torch.ones(500, dtype=torch.float64, device="cuda")
    y_d = torch.zeros(500, dtype=torch.float64, device="cuda")
    assert _noalloc(1, 500, 500, rp_d, col_d, val_d, x_d, y_d) == getattr(_lib, status), name
    # the status word is cleared by the next call: a valid matrix right after works
    grp, gcol, gval = rand_crs(500, 10, 28)
    x = rng.uniform(-1, 1, 500)
    y = _run_noalloc(grp, gcol, gval, x, 500)
    assert normwise(y, _oracle_y(grp, gcol, gval, x)) <= 1e-12
