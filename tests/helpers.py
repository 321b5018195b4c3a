"""Shared helpers of the parity tests: tolerances, random CRS matrices and thin
wrappers that run one kernel through the Python mirror of SMAX::Interface."""
from __future__ import annotations

import numpy as np

# Normwise relative tolerances against the reference's OpenMP output
# (FP64: 1e-12, FP32: 1e-5), each also stated against an FP64 oracle.
TOL = {np.float64: 1e-12, np.float32: 1e-5}


def tol(dtype) -> float:
    return TOL[np.float32] if np.dtype(dtype) == np.float32 else TOL[np.float64]


def normwise(got, ref) -> float:
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    d = np.linalg.norm(got - ref)
    r = np.linalg.norm(ref)
    return float(d / r) if r > 0 else float(d)


def rand_crs(n, maxlen, seed, vt=np.float64, n_cols=None, empty_frac=0.0, long_rows=(), lower=False):
    """Random CRS matrix with sorted unique columns; optional empty rows and
    a few very long rows (length given in long_rows)."""
    rng = np.random.default_rng(seed)
    n_cols = n_cols or n
    lens = rng.integers(0, maxlen + 1, n)
    if empty_frac:
        lens[rng.random(n) < empty_frac] = 0
    for i, L in enumerate(long_rows):
        lens[(i * 7919) % max(n, 1)] = min(L, n_cols)
    rows = []
    for r in range(n):
        if lower:
            k = int(min(lens[r], r))
            c = np.concatenate([rng.choice(r, k, replace=False) if k else np.zeros(0, np.int64), [r]])
        else:
            c = rng.choice(n_cols, int(lens[r]), replace=False) if lens[r] else np.zeros(0, np.int64)
        rows.append(np.sort(c))
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(c) for c in rows])
    col = (np.concatenate(rows) if rows else np.zeros(0)).astype(np.int32)
    val = rng.uniform(-1, 1, len(col)).astype(vt)
    if lower:
        val[rp[1:] - 1] = (4.0 + rng.uniform(0, 1, n)).astype(vt)
    return rp, col, val


def gpu_spmv(row_ptr, col, val, x, n_cols=None, variant=0):
    from smaxkernels_b200 import FloatType, Interface, KernelType, PlatformType, IntType
    ft = FloatType.FLOAT32 if val.dtype == np.float32 else FloatType.FLOAT64
    n = len(row_ptr) - 1
    y = np.zeros(n, dtype=val.dtype)
    smax = Interface()
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, ft)
    k = smax.kernel("k")
    if variant:
        k.set_spmv_variant(variant)
    k.register_A(n, n_cols or len(x), len(col), col, row_ptr, val)
    k.register_B(len(x), np.ascontiguousarray(x, dtype=val.dtype))
    k.register_C(n, y)
    k.run()
    smax.close()
    return y
