"""Parity at the timed configurations against the reference itself.

Every other config-size GPU test compares the CUDA result with the plain-C
restatement (liboracle.so).  These tests compare it directly with the
unmodified reference, compiled from its own sources into
oracle/_ref/libsmax_ref.so and run through its SMAX::Interface on the host's
cores (its OpenMP kernels: the `omp simd` CRS loop, the reference's SELL-C-
sigma and BCRS conversions, its Gustavson SpGEMM, level-scheduled SpTRSV and
permutations), on the same seeded inputs:

  config 0  CRS SpMV, 7-point 64^3 Laplacian                FP64, FP32
  config 1  CRS SpMV, lognormal 2^22 rows (nnz 67.2 M)      FP64, FP32
            SELL-32-1024 conversion + SpMV                  FP64, FP32
            BCRS 4x4 conversion + SpMV, both in-block orders FP64
  config 2  SpMM, 27-point 128^3 stencil, k = 16 and 64     FP64, FP32
            SpGEMM C = A*A, 7-point 96^3 (pattern bit-exact) FP64
  config 3  SpTRSV, lower 5-point 2048^2, natural order     FP64
            SpTRSV, seed-3 random symmetric permutation, RS levels (perm,
            levels and permuted matrix bit-exact)           FP64
            SpTRSM k = 32, natural order                    FP64
            generate_perm RS and BFS on the 2048^2 grid (BFS against the
            reference run on one thread, where its queue order is defined)

Tolerances: normwise relative 1e-12 (FP64) and 1e-5 (FP32) against the
reference's own output in the same precision; FP32 results are also held to
1e-5 against the reference's FP64 output.  Integer arrays are bit-exact,
including the SELL-C-sigma permutation at sigma = 1024: the reference orders
rows of equal length inside a sigma window the way its std::sort leaves them,
and the GPU conversion reproduces that order (csrc/scs_window_sort.cuh), so
perm, col and val match the reference's entry for entry.
"""
import os

import numpy as np
import pytest

from helpers import gpu_spmv, normwise, tol
from oracle.oracle import Reference, reference_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not reference_available(),
                                                  reason="oracle/_ref/libsmax_ref.so is not built")]

_R = None


def R():
    global _R
    if _R is None:
        _R = Reference()
        _R.set_threads(os.cpu_count() or 1)
    return _R


def _M():
    from smaxkernels_b200 import matrices as M
    return M


def _iface():
    from smaxkernels_b200 import Interface
    return Interface()


def _ft(vt):
    from smaxkernels_b200 import FloatType
    return FloatType.FLOAT32 if np.dtype(vt) == np.float32 else FloatType.FLOAT64


def _check_fp(got, ref, vt, ref64=None, what=""):
    assert normwise(got, ref) <= tol(vt), f"{what}: {normwise(got, ref):.3e} against the reference"
    if ref64 is not None:
        assert normwise(got, ref64) <= tol(vt), f"{what}: {normwise(got, ref64):.3e} against the FP64 reference"


# ------------------------------------------------------------------ CRS ----
@pytest.mark.parametrize("vt", [np.float64, np.float32])
def test_crs_config0_vs_reference(vt):
    M = _M()
    rp, col, val64 = M.laplace3d_7pt(64)
    n = len(rp) - 1
    x64 = M.uniform_vector(n, 0)
    val, x = val64.astype(vt), x64.astype(vt)
    y = gpu_spmv(rp, col, val, x)
    ref64 = R().spmv_crs(rp, col, val64, x64) if vt == np.float32 else None
    _check_fp(y, R().spmv_crs(rp, col, val, x), vt, ref64, "config 0 CRS")


@pytest.mark.slow
@pytest.mark.parametrize("vt", [np.float64, np.float32])
def test_crs_config1_vs_reference(vt):
    M = _M()
    rp, col, val64 = M.lognormal_random(1 << 22, seed=1)
    n = len(rp) - 1
    x64 = M.uniform_vector(n, 100)
    val, x = val64.astype(vt), x64.astype(vt)
    y = gpu_spmv(rp, col, val, x)
    ref64 = R().spmv_crs(rp, col, val64, x64) if vt == np.float32 else None
    _check_fp(y, R().spmv_crs(rp, col, val, x), vt, ref64, "config 1 CRS")


# --------------------------------------------------------- SELL-C-sigma ----
def _gpu_scs_spmv(s, x):
    from smaxkernels_b200 import IntType, KernelType, PlatformType
    vt = s["val"].dtype
    vs = max(s["n_rows_padded"], len(x))
    xx = np.zeros(vs, dtype=vt)
    xx[: len(x)] = x
    y = np.zeros(vs, dtype=vt)
    smax = _iface()
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, _ft(vt))
    k = smax.kernel("k")
    k.set_mat_scs(True)
    k.register_A(s["C"], s["sigma"], s["n_rows"], s["n_rows_padded"], len(x), s["n_chunks"], s["n_elements"],
                 s["nnz"], s["chunk_ptr"], s["chunk_lengths"], s["col"], s["val"], s["perm"])
    k.register_B(vs, xx)
    k.register_C(vs, y)
    k.run()
    smax.close()
    return y


def assert_same_scs(got, ref):
    """Two SELL-C-sigma conversions of one matrix are identical."""
    for key in ("n_rows", "n_rows_padded", "n_chunks", "n_elements", "nnz"):
        assert got[key] == ref[key], key
    for key in ("chunk_ptr", "chunk_lengths", "perm", "col", "val"):
        np.testing.assert_array_equal(got[key], ref[key], err_msg=key)


@pytest.mark.slow
@pytest.mark.parametrize("vt", [np.float64, np.float32])
def test_scs_config1_vs_reference(vt):
    M = _M()
    rp, col, val64 = M.lognormal_random(1 << 22, seed=1)
    n = len(rp) - 1
    val = val64.astype(vt)
    x64 = M.uniform_vector(n, 1)
    x = x64.astype(vt)
    smax = _iface()
    got = smax.utils.convert_crs_to_scs(n, n, len(col), col, rp, val, 32, 1024)
    smax.close()
    ref = R().scs(rp, col, val, 32, 1024)
    assert_same_scs(got, ref)  # the window order of equal-length rows included
    # the GPU kernel on the REFERENCE's own arrays gives the reference's y
    y_on_ref_layout = _gpu_scs_spmv(ref, x)
    y_ref = R().spmv_scs(ref, x)
    _check_fp(y_on_ref_layout[: ref["n_rows_padded"]], y_ref[: ref["n_rows_padded"]], vt, None,
              "SELL SpMV on the reference's layout")
    # and the whole GPU flow (GPU conversion + kernel), un-permuted, matches too
    y_gpu = _gpu_scs_spmv(got, x)
    ref64 = None
    if vt == np.float32:
        r64 = R().scs(rp, col, val64, 32, 1024)
        ref64 = R().spmv_scs(r64, x64)[r64["perm"]]
    _check_fp(y_gpu[got["perm"]], y_ref[ref["perm"]], vt, ref64, "SELL SpMV after un-permuting")


# ------------------------------------------------------------------ BCRS ----
@pytest.mark.slow
@pytest.mark.parametrize("col_major", [False, True])
def test_bcrs4x4_config1_vs_reference(col_major):
    """4x4 BCRS of the 2^22 lognormal matrix (n_blocks ~ nnz, 8.6 GB of FP64
    block values): the GPU conversion is bit-exact with the reference's, and
    the GPU SpMV on it matches the reference's SpMV."""
    from smaxkernels_b200 import IntType, KernelType, PlatformType
    M = _M()
    rp, col, val = M.lognormal_random(1 << 22, seed=1)
    n = len(rp) - 1
    x = M.uniform_vector(n, 1)
    ref = R().bcrs(rp, col, val, n, 4, 4, 4, 4, col_major)
    y_ref = R().spmv_bcrs(ref, x, col_major)
    smax = _iface()
    got = smax.utils.convert_crs_to_bcrs(n, n, len(col), col, rp, val, 4, 4, 4, 4, col_major)
    for key in ("n_rows", "n_cols", "n_blocks"):
        assert got[key] == ref[key], key
    for key in ("row_ptr", "col", "val"):
        assert np.array_equal(got[key], ref[key]), key
    del ref
    y = np.zeros(got["n_rows"] * 4)
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, _ft(np.float64))
    k = smax.kernel("k")
    k.set_mat_bcrs(True)
    k.register_A(got["n_rows"], got["n_cols"], got["n_blocks"], 4, 4, 4, 4, got["col"], got["row_ptr"], got["val"])
    k.register_B(n, x)
    k.register_C(n, y)
    k.set_block_column_major(col_major)
    k.run()
    smax.close()
    _check_fp(y, y_ref, np.float64, None, f"BCRS 4x4 col_major={col_major}")


# ------------------------------------------------------------------ SpMM ----
@pytest.mark.slow
@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("k_", [16, 64])
def test_spmm_config2_vs_reference(vt, k_):
    from smaxkernels_b200 import IntType, KernelType, PlatformType
    M = _M()
    rp, col, val64 = M.stencil27(128)
    n = len(rp) - 1
    X64 = np.random.default_rng(2).uniform(-1, 1, n * k_)
    val, X = val64.astype(vt), X64.astype(vt)
    Y = np.zeros(n * k_, dtype=vt)
    smax = _iface()
    smax.register_kernel("k", KernelType.SPMM, PlatformType.CUDA, IntType.INT32, _ft(vt))
    k = smax.kernel("k")
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, k_, X)
    k.register_C(n, k_, Y)
    k.set_vec_row_major(True)
    k.run()
    smax.close()
    ref64 = R().spmm(rp, col, val64, X64, k_, row_major=True) if vt == np.float32 else None
    _check_fp(Y, R().spmm(rp, col, val, X, k_, row_major=True), vt, ref64, f"SpMM k={k_}")


# ---------------------------------------------------------------- SpGEMM ----
@pytest.mark.slow
@pytest.mark.parametrize("vt", [np.float64, np.float32])
def test_spgemm_config2_vs_reference(vt):
    """Two runs on one kernel object: the first classifies the rows, the
    second takes the direct merge path at once.  Both equal the reference."""
    from smaxkernels_b200 import IntType, KernelType, PlatformType
    M = _M()
    rp, col, val64 = M.laplace3d_7pt(96)
    val = val64.astype(vt)
    n = len(rp) - 1
    orp, ocol, oval, onr, onc = R().spgemm(rp, col, val, rp, col, val, n, n)
    ref64 = R().spgemm(rp, col, val64, rp, col, val64, n, n)[2] if vt == np.float32 else None
    smax = _iface()
    smax.register_kernel("g", KernelType.SPGEMM, PlatformType.CUDA, IntType.INT32, _ft(vt))
    k = smax.kernel("g")
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, n, len(col), col, rp, val)
    for run in range(2):
        k.register_C()
        k.run()
        n_rows, n_cols, nnz, crp, ccol, cval = k.result()
        assert (n_rows, n_cols, nnz) == (onr, onc, len(ocol)) and nnz == 21_732_480
        np.testing.assert_array_equal(crp, orp)
        np.testing.assert_array_equal(ccol, ocol)  # first-touch order inside every row
        _check_fp(cval, oval, vt, ref64, f"SpGEMM values, run {run}")
    smax.close()


# ------------------------------------------------------ SpTRSV / SpTRSM ----
def _gpu_tri(rp, col, val, b, levels=None, k_=None):
    """SpTRSV (SpTRSM with k_ columns) through the Interface; with `levels`,
    the matrix is level-permuted and these are its level pointers
    (set_mat_perm(true), as the reference's level-scheduled flow)."""
    from smaxkernels_b200 import IntType, KernelType, PlatformType
    n = len(rp) - 1
    smax = _iface()
    if levels is not None:
        smax.set_levels(levels)
    kt = KernelType.SPTRSM if k_ else KernelType.SPTRSV
    smax.register_kernel("t", kt, PlatformType.CUDA, IntType.INT32, _ft(val.dtype))
    k = smax.kernel("t")
    if levels is not None:
        k.set_mat_perm(True)
    c, v = col.copy(), val.copy()
    k.register_A(n, n, len(c), c, rp, v)
    if k_:
        x = np.zeros(n * k_, val.dtype)
        k.register_B(n, k_, x)
        k.register_C(n, k_, np.ascontiguousarray(b, val.dtype))
        k.set_vec_row_major(True)
    else:
        x = np.zeros(n, val.dtype)
        k.register_B(n, x)
        k.register_C(n, np.ascontiguousarray(b, val.dtype))
    k.run()
    smax.close()
    return x


@pytest.mark.slow
def test_sptrsv_config3_natural_vs_reference():
    M = _M()
    lrp, lcol, lval = M.lower_triangle(*M.laplace2d_5pt(2048))
    b = M.uniform_vector(len(lrp) - 1, 3)
    x = _gpu_tri(lrp, lcol, lval, b)
    _check_fp(x, R().sptrsv(lrp, lcol, lval, b), np.float64, None, "natural SpTRSV")


def _gpu_perm(rp, col, type_):
    smax = _iface()
    n = len(rp) - 1
    perm = np.zeros(n, np.int32)
    inv = np.zeros(n, np.int32)
    smax.utils.generate_perm(n, rp, col, perm, inv, type_)
    lvl = np.array([smax.get_level_ptr_at(i) for i in range(smax.get_n_levels() + 1)], np.int32)
    smax.close()
    return perm, inv, lvl


def _ref_perm_one_thread(rp, col, type_):
    """The reference's generate_perm on one thread: its BFS queue order is
    only defined there (permutations.hpp:416-483 appends under OpenMP)."""
    r = R()
    r.set_threads(1)
    try:
        return r.generate_perm(rp, col, type_)
    finally:
        r.set_threads(os.cpu_count() or 1)


@pytest.mark.slow
@pytest.mark.parametrize("grid", ["natural", "permuted"])
@pytest.mark.parametrize("type_", ["RS", "BFS"])
def test_generate_perm_2048_vs_reference(grid, type_):
    M = _M()
    A = M.laplace2d_5pt(2048)
    if grid == "permuted":
        A = M.random_symmetric_permutation(*A, seed=3)[:3]
    rp, col = A[0], A[1]
    perm, inv, lvl = _gpu_perm(rp, col, type_)
    rperm, rinv, rlvl = _ref_perm_one_thread(rp, col, type_)
    np.testing.assert_array_equal(lvl, rlvl)
    np.testing.assert_array_equal(perm, rperm)
    np.testing.assert_array_equal(inv, rinv)


@pytest.mark.slow
def test_sptrsv_config3_permuted_vs_reference():
    """The reference's level-scheduled flow on the seed-3 permuted 2048^2 grid
    (examples/demos/sptrsv_lvl_demo.cpp:69-116): RS levels, apply_mat_perm,
    lower triangle, set_mat_perm(true).  Every integer step is bit-exact with
    the reference's; the solve matches its level-scheduled solve."""
    M = _M()
    Ar, Ac, Av, _ = M.random_symmetric_permutation(*M.laplace2d_5pt(2048), seed=3)
    n = len(Ar) - 1
    smax = _iface()
    perm = np.zeros(n, np.int32)
    inv = np.zeros(n, np.int32)
    smax.utils.generate_perm(n, Ar, Ac, perm, inv, "RS")
    lvl = np.array([smax.get_level_ptr_at(i) for i in range(smax.get_n_levels() + 1)], np.int32)
    prp = np.zeros(n + 1, np.int32)
    pcol = np.zeros(len(Ac), np.int32)
    pval = np.zeros(len(Ac))
    smax.utils.apply_mat_perm(n, Ar, Ac, Av, prp, pcol, pval, perm, inv)
    smax.close()
    rperm, rinv, rlvl = R().generate_perm(Ar, Ac, "RS")
    np.testing.assert_array_equal(perm, rperm)
    np.testing.assert_array_equal(lvl, rlvl)
    rrp, rcol, rval = R().apply_mat_perm(Ar, Ac, Av, rperm, rinv)
    np.testing.assert_array_equal(prp, rrp)
    np.testing.assert_array_equal(pcol, rcol)
    np.testing.assert_array_equal(pval, rval)
    lrp, lcol, lval = M.lower_triangle(prp, pcol, pval)
    b = M.uniform_vector(n, 3)
    x = _gpu_tri(lrp, lcol, lval, b, levels=lvl)
    _check_fp(x, R().sptrsv(lrp, lcol, lval, b, levels=lvl), np.float64, None, "permuted level-scheduled SpTRSV")


@pytest.mark.slow
def test_sptrsm_config3_k32_vs_reference():
    M = _M()
    lrp, lcol, lval = M.lower_triangle(*M.laplace2d_5pt(2048))
    n = len(lrp) - 1
    B = np.random.default_rng(3).uniform(-1, 1, n * 32)
    X = _gpu_tri(lrp, lcol, lval, B, k_=32)
    _check_fp(X, R().sptrsm(lrp, lcol, lval, B, 32, row_major=True), np.float64, None, "SpTRSM k=32")
