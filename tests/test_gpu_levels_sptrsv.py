"""Parity of the GPU level sets, permutations, SpTRSV and SpTRSM with the
oracle and the reference's golden vectors (through the C ABI)."""
import numpy as np
import pytest

import golden_cases as G
from helpers import normwise, rand_crs, tol
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
O = Oracle()


def _iface():
    from smaxkernels_b200 import Interface
    return Interface()


def _ft(vt):
    from smaxkernels_b200 import FloatType
    return FloatType.FLOAT32 if np.dtype(vt) == np.float32 else FloatType.FLOAT64


def gpu_perm(rp, col, type_):
    smax = _iface()
    n = len(rp) - 1
    perm = np.zeros(n, np.int32)
    inv = np.zeros(n, np.int32)
    smax.utils.generate_perm(n, rp, col, perm, inv, type_)
    lvl = np.array([smax.get_level_ptr_at(i) for i in range(smax.get_n_levels() + 1)], np.int32)
    smax.close()
    return perm, inv, lvl


def gpu_sptrsv(rp, col, val, b, upper=False, mode=0, merge=-1, sptrsm_k=None, row_major=True):
    """Runs SpTRSV (or SpTRSM with sptrsm_k columns) like the reference tests do;
    returns (x, col_after, val_after) -- the registered arrays are mutated."""
    from smaxkernels_b200 import IntType, KernelType, PlatformType
    col = col.copy()
    val = val.copy()
    n = len(rp) - 1
    smax = _iface()
    kt = KernelType.SPTRSM if sptrsm_k else KernelType.SPTRSV
    smax.register_kernel("k", kt, PlatformType.CUDA, IntType.INT32, _ft(val.dtype))
    k = smax.kernel("k")
    if upper:
        k.set_mat_upper_triang(True)
    if mode:
        k.set_solve_mode(mode)
    if merge >= 0:
        k.set_level_merge(merge)
    k.register_A(n, n, len(col), col, rp, val)
    if sptrsm_k:
        x = np.zeros(n * sptrsm_k, val.dtype)
        k.register_B(n, sptrsm_k, x)
        k.register_C(n, sptrsm_k, np.ascontiguousarray(b, val.dtype))
        k.set_vec_row_major(row_major)
    else:
        x = np.zeros(n, val.dtype)
        k.register_B(n, x)
        k.register_C(n, np.ascontiguousarray(b, val.dtype))
    k.run()
    smax.close()
    return x, col, val


# ------------------------------------------------------------- A + A^T ----
@pytest.mark.parametrize("name", ["build_symmetric_crs_1", "build_symmetric_crs_2", "build_symmetric_crs_3"])
def test_build_symmetric_golden_on_gpu(name):
    c = G.symmetric_case(name)
    smax = _iface()
    srp, scol, nz = smax.utils.build_symmetric_crs(c["row_ptr"], c["col"], len(c["row_ptr"]) - 1)
    smax.close()
    np.testing.assert_array_equal(srp, c["sym_row_ptr"])
    np.testing.assert_array_equal(G.sort_rows(srp, scol), c["sym_col"])
    # and the exact in-row order of the reference (one-thread append order)
    orp, ocol = O.build_symmetric(c["row_ptr"], c["col"])
    np.testing.assert_array_equal(scol, ocol)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_build_symmetric_random(seed):
    rp, col, val = rand_crs(700, 12, seed, empty_frac=0.2)
    smax = _iface()
    srp, scol, nz = smax.utils.build_symmetric_crs(rp, col, 700)
    smax.close()
    orp, ocol = O.build_symmetric(rp, col)
    np.testing.assert_array_equal(srp, orp)
    np.testing.assert_array_equal(scol, ocol)


# ------------------------------------------------------- permutations ----
@pytest.mark.parametrize("name", ["perm_test_1", "perm_test_2"])
def test_perm_golden_on_gpu(name):
    c = G.perm_case(name)
    for typ, exp_perm, exp_val in (("BFS", c["perm_bfs"], c["val_bfs"]), ("RS", c["perm_rs"], c["val_rs"])):
        perm, inv, lvl = gpu_perm(c["row_ptr"], c["col"], typ)
        assert len(lvl) - 1 == c["n_levels"]
        np.testing.assert_array_equal(lvl, c["lvl_ptr"])
        np.testing.assert_array_equal(perm, exp_perm)
        np.testing.assert_array_equal(perm[inv], np.arange(len(perm)))
        n = len(perm)
        prp = np.zeros(n + 1, np.int32)
        pcol = np.zeros(len(c["col"]), np.int32)
        pval = np.zeros(len(c["col"]))
        smax = _iface()
        smax.utils.apply_mat_perm(n, c["row_ptr"], c["col"], c["val"], prp, pcol, pval, perm, inv)
        smax.close()
        np.testing.assert_array_equal(pval, exp_val)
        orp, ocol, oval = O.apply_mat_perm(c["row_ptr"], c["col"], c["val"], perm, inv)
        np.testing.assert_array_equal(prp, orp)
        np.testing.assert_array_equal(pcol, ocol)


@pytest.mark.parametrize("typ", ["BFS", "RS", "NONE"])
@pytest.mark.parametrize("kind", ["lower", "general", "empty_rows"])
def test_perm_random_vs_oracle(typ, kind):
    if kind == "lower":
        rp, col, val = rand_crs(2000, 6, 61, lower=True)
    elif kind == "general":
        rp, col, val = rand_crs(2000, 8, 62)
    else:
        rp, col, val = rand_crs(2000, 5, 63, empty_frac=0.6)
    perm, inv, lvl = gpu_perm(rp, col, typ)
    operm, oinv, olvl = O.generate_perm(rp, col, typ)
    np.testing.assert_array_equal(lvl, olvl)
    np.testing.assert_array_equal(perm, operm)
    np.testing.assert_array_equal(inv, oinv)


@pytest.mark.slow
@pytest.mark.parametrize("typ", ["BFS", "RS"])
def test_perm_laplace2d(typ):
    """Wide levels (grid-wide sweep) and long level chains (single-CTA sweep)."""
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace2d_5pt(300)
    prp, pcol, pval, _ = M.random_symmetric_permutation(rp, col, val, seed=3)
    for (a, b) in ((rp, col), (prp, pcol)):
        perm, inv, lvl = gpu_perm(a, b, typ)
        operm, oinv, olvl = O.generate_perm(a, b, typ)
        np.testing.assert_array_equal(lvl, olvl)
        np.testing.assert_array_equal(perm, operm)


def test_perm_unknown_type():
    from smaxkernels_b200 import SmaxError
    rp, col, val = rand_crs(50, 4, 1)
    with pytest.raises(SmaxError, match="does not exist"):
        gpu_perm(rp, col, "XYZ")


def test_apply_vec_perm():
    v = np.random.default_rng(1).uniform(-1, 1, 1000)
    perm = np.random.default_rng(2).permutation(1000).astype(np.int32)
    out = np.zeros(1000)
    smax = _iface()
    smax.utils.apply_vec_perm(1000, v, out, perm)
    smax.close()
    np.testing.assert_array_equal(out, O.apply_vec_perm(v, perm))


# ------------------------------------------------------------------ SpTRSV --
def test_sptrsv_golden():
    c = G.sptrsv_case()
    x, _, _ = gpu_sptrsv(c["row_ptr"], c["col"], c["val"], c["b"])
    assert G.almost_equal(x, c["x"], np.float64)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("mode,merge", [(0, -1), (1, -1), (2, 0), (2, 64), (3, 4096), (3, 1)])
def test_sptrsv_random_plain_vs_oracle(vt, upper, mode, merge):
    rp, col, val = rand_crs(3000, 8, 71, vt=vt, lower=True)
    if upper:  # transpose the lower triangle into an upper one (diagonal first in each row)
        import scipy.sparse as sp
        L = sp.csr_matrix((val, col, rp), shape=(3000, 3000))
        U = L.T.tocsr()
        U.sort_indices()
        rp, col, val = U.indptr.astype(np.int32), U.indices.astype(np.int32), U.data.astype(vt)
    b = np.random.default_rng(72).uniform(-1, 1, 3000).astype(vt)
    x, col_after, val_after = gpu_sptrsv(rp, col, val, b, upper=upper, mode=mode, merge=merge)
    x_ref = O.sptrsv(rp, col, val, b, lower=not upper)
    assert normwise(x, x_ref) <= tol(vt)
    # the registered arrays carry the diagonal at the end of each row afterwards
    pcol, pval, _ = O.peel_diag(rp, col, val)
    np.testing.assert_array_equal(col_after, pcol)
    np.testing.assert_array_equal(val_after, pval)


def test_sptrsv_level_scheduled_reference_flow():
    """generate_perm -> apply_mat_perm -> lower triangle -> set_mat_perm(true)
    (examples/demos/sptrsv_lvl_demo.cpp:69-116), through one Interface."""
    from smaxkernels_b200 import FloatType, IntType, KernelType, PlatformType
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace2d_5pt(120)
    n = len(rp) - 1
    for typ in ("RS", "BFS"):
        smax = _iface()
        perm = np.zeros(n, np.int32)
        inv = np.zeros(n, np.int32)
        smax.utils.generate_perm(n, rp, col, perm, inv, typ)
        prp = np.zeros(n + 1, np.int32)
        pcol = np.zeros(len(col), np.int32)
        pval = np.zeros(len(col))
        smax.utils.apply_mat_perm(n, rp, col, val, prp, pcol, pval, perm, inv)
        lrp, lcol, lval = M.lower_triangle(prp, pcol, pval)
        b = np.random.default_rng(5).uniform(-1, 1, n)
        x = np.zeros(n)
        lcol_reg, lval_reg = lcol.copy(), lval.copy()
        for mode in (1, 2, 3):
            smax.register_kernel("tri", KernelType.SPTRSV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
            k = smax.kernel("tri")
            k.set_mat_perm(True)
            k.set_solve_mode(mode)
            k.register_A(n, n, len(lcol_reg), lcol_reg, lrp, lval_reg)
            k.register_B(n, x)
            k.register_C(n, b)
            k.run()
            lvl = np.array([smax.get_level_ptr_at(i) for i in range(smax.get_n_levels() + 1)], np.int32)
            x_ref = O.sptrsv(lrp, lcol, lval, b, levels=lvl)
            assert normwise(x, x_ref) <= 1e-12, (typ, mode)
        smax.close()


@pytest.mark.parametrize("vt", [np.float64, np.float32])
def test_sptrsv_level_scheduled_upper_descending(vt):
    """Upper solve on permuted levels walks the levels from last to first
    (src/kernels/sptrsv/sptrsv_cpu/sptrsv_lvl_cpu_crs_impl.hpp:51)."""
    from smaxkernels_b200 import IntType, KernelType, PlatformType
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace2d_5pt(60, dtype=vt)
    n = len(rp) - 1
    smax = _iface()
    perm = np.zeros(n, np.int32)
    inv = np.zeros(n, np.int32)
    smax.utils.generate_perm(n, rp, col, perm, inv, "RS")
    prp = np.zeros(n + 1, np.int32)
    pcol = np.zeros(len(col), np.int32)
    pval = np.zeros(len(col), vt)
    smax.utils.apply_mat_perm(n, rp, col, val, prp, pcol, pval, perm, inv)
    # upper part incl. diagonal
    row = np.repeat(np.arange(n), np.diff(prp))
    keep = pcol >= row
    urp = np.zeros(n + 1, np.int32)
    urp[1:] = np.cumsum(np.bincount(row[keep], minlength=n))
    ucol, uval = pcol[keep].copy(), pval[keep].copy()
    b = np.random.default_rng(6).uniform(-1, 1, n).astype(vt)
    x = np.zeros(n, vt)
    smax.register_kernel("tri", KernelType.SPTRSV, PlatformType.CUDA, IntType.INT32, _ft(vt))
    k = smax.kernel("tri")
    k.set_mat_perm(True)
    k.set_mat_upper_triang(True)
    k.register_A(n, n, len(ucol), ucol.copy(), urp, uval.copy())
    k.register_B(n, x)
    k.register_C(n, b)
    k.run()
    lvl = np.array([smax.get_level_ptr_at(i) for i in range(smax.get_n_levels() + 1)], np.int32)
    smax.close()
    x_ref = O.sptrsv(urp, ucol, uval, b, lower=False, levels=lvl)
    assert normwise(x, x_ref) <= tol(vt)


@pytest.mark.parametrize("bad", ["zero", "missing"])
def test_sptrsv_bad_diagonal_is_an_error(bad):
    from smaxkernels_b200 import SmaxError, _lib
    rp, col, val = rand_crs(100, 4, 81, lower=True)
    val = val.copy()
    rp = rp.copy()
    col = col.copy()
    if bad == "zero":
        val[rp[50 + 1] - 1] = 0.0
        code = _lib.ERR_ZERO_DIAG
    else:
        col[rp[51] - 1] = 49  # row 50 loses its diagonal entry
        code = _lib.ERR_NO_DIAG
    with pytest.raises(SmaxError) as e:
        gpu_sptrsv(rp, col, val, np.ones(100))
    assert e.value.code == code


@pytest.mark.slow
def test_sptrsv_config3_natural_2048():
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace2d_5pt(2048)
    lrp, lcol, lval = M.lower_triangle(rp, col, val)
    b = M.uniform_vector(len(lrp) - 1, 3)
    x, _, _ = gpu_sptrsv(lrp, lcol, lval, b)
    x_ref = O.sptrsv(lrp, lcol, lval, b)
    assert normwise(x, x_ref) <= 1e-12


# ------------------------------------------------------------------ SpTRSM --
@pytest.mark.parametrize("name", ["sptrsm_test", "sptrsm_rowmaj_test"])
def test_sptrsm_golden(name):
    c = G.sptrsm_case(name)
    X, _, _ = gpu_sptrsv(c["row_ptr"], c["col"], c["val"], c["B"], sptrsm_k=c["k"], row_major=c["row_major"])
    assert G.almost_equal(X, c["X"], np.float64)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("k_", [1, 3, 32])
@pytest.mark.parametrize("row_major", [True, False])
@pytest.mark.parametrize("mode", [1, 3])
def test_sptrsm_random_vs_oracle(vt, k_, row_major, mode):
    rp, col, val = rand_crs(1500, 6, 91, vt=vt, lower=True)
    B = np.random.default_rng(92).uniform(-1, 1, 1500 * k_).astype(vt)
    X, _, _ = gpu_sptrsv(rp, col, val, B, sptrsm_k=k_, row_major=row_major, mode=mode)
    X_ref = O.sptrsm(rp, col, val, B, k_, row_major=row_major)
    assert normwise(X, X_ref) <= tol(vt)


def test_sptrsv_level_scheduled_with_levels_from_the_oracle():
    """Levels computed on the CPU (the reference's generate_perm restated by the
    oracle) handed over with set_levels drive the level-scheduled solve."""
    from smaxkernels_b200 import FloatType, IntType, KernelType, PlatformType
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace2d_5pt(90)
    n = len(rp) - 1
    perm, inv, lvl = O.generate_perm(rp, col, "RS")
    prp, pcol, pval = O.apply_mat_perm(rp, col, val, perm, inv)
    lrp, lcol, lval = M.lower_triangle(prp, pcol, pval)
    smax = _iface()
    smax.set_levels(lvl)
    assert smax.get_n_levels() == len(lvl) - 1
    smax.register_kernel("tri", KernelType.SPTRSV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("tri")
    k.set_mat_perm(True)
    b = np.random.default_rng(21).uniform(-1, 1, n)
    x = np.zeros(n)
    k.register_A(n, n, len(lcol), lcol.copy(), lrp, lval.copy())
    k.register_B(n, x)
    k.register_C(n, b)
    k.run()
    assert normwise(x, O.sptrsv(lrp, lcol, lval, b, levels=lvl)) <= 1e-12
    smax.close()
