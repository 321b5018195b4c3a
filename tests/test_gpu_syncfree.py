"""Sync-free triangular solve (SMAX_SOLVE_SYNCFREE): one launch in which each
row waits on the rows it reads instead of a barrier per level.  The per-row
arithmetic is the level kernels' (off-diagonal products summed in stored
order, then (b - sum) * (1 / D)), so results are compared bit for bit with
the merged solve, and with the oracle's restatement of the reference's
naive_crs_sptrsv / crs_sptrsv_lvl
(src/kernels/sptrsv/sptrsv_cpu/sptrsv_cpu_crs_impl.hpp:9-55,
sptrsv_lvl_cpu_crs_impl.hpp:11-82)."""
import numpy as np
import pytest

from helpers import normwise, rand_crs, tol
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
O = Oracle()

SYNCFREE, MERGED = 5, 2


def _solve(rp, col, val, b, mode, upper=False, perm_levels=None, spin=None, force_timeout=False):
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    n = len(rp) - 1
    smax = Interface()
    if perm_levels is not None:
        smax.set_levels(perm_levels)
    smax.register_kernel("t", KernelType.SPTRSV, PlatformType.CUDA, IntType.INT32,
                         FloatType.FLOAT64 if val.dtype == np.float64 else FloatType.FLOAT32)
    k = smax.kernel("t")
    k.set_solve_mode(mode)
    if mode == MERGED:
        k.set_level_merge(0)
    if perm_levels is not None:
        k.set_mat_perm(True)
    if upper:
        k.set_mat_upper_triang(True)
    if spin:
        k.set_spin_limit(spin)
    if force_timeout:
        k._flag("test_force_timeout", 1)
    x = np.zeros(n, val.dtype)
    k.register_A(n, n, len(col), col.copy(), rp, val.copy())
    k.register_B(n, x)
    k.register_C(n, np.ascontiguousarray(b, val.dtype))
    return smax, k, x


def _run(*a, **kw):
    smax, k, x = _solve(*a, **kw)
    k.run()
    smax.close()
    return x


def _upper(rp, col, val):
    import scipy.sparse as sp
    n = len(rp) - 1
    U = sp.csr_matrix((val, col, rp), shape=(n, n)).T.tocsr()
    U.sort_indices()
    return U.indptr.astype(np.int32), U.indices.astype(np.int32), U.data.astype(val.dtype)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("n,per_row,seed", [(3000, 8, 71), (20000, 3, 5), (777, 40, 9)])
def test_syncfree_vs_oracle_and_merged(vt, upper, n, per_row, seed):
    rp, col, val = rand_crs(n, per_row, seed, vt=vt, lower=True)
    if upper:
        rp, col, val = _upper(rp, col, val)
    b = np.random.default_rng(seed + 1).uniform(-1, 1, n).astype(vt)
    x = _run(rp, col, val, b, SYNCFREE, upper=upper)
    assert normwise(x, O.sptrsv(rp, col, val, b, lower=not upper)) <= tol(vt)
    np.testing.assert_array_equal(x, _run(rp, col, val, b, MERGED, upper=upper))


@pytest.mark.parametrize("side", [64, 300])
def test_syncfree_laplace_natural(side):
    """Thousands of one-row-wide dependency chains: every level waits on the last."""
    from smaxkernels_b200 import matrices as M
    lrp, lcol, lval = M.lower_triangle(*M.laplace2d_5pt(side))
    b = M.uniform_vector(len(lrp) - 1, 3)
    x = _run(lrp, lcol, lval, b, SYNCFREE)
    assert normwise(x, O.sptrsv(lrp, lcol, lval, b)) <= 1e-12
    np.testing.assert_array_equal(x, _run(lrp, lcol, lval, b, MERGED))


@pytest.mark.parametrize("upper", [False, True])
def test_syncfree_level_scheduled_flow(upper):
    """generate_perm(RS) -> apply_mat_perm -> triangle -> set_mat_perm(true),
    the permuted flow of examples/demos/sptrsv_lvl_demo.cpp:69-116; the upper
    triangle sweeps its levels last to first."""
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace2d_5pt(150)
    n = len(rp) - 1
    Ar, Ac, Av, _ = M.random_symmetric_permutation(rp, col, val, seed=3)
    perm, inv, lvl = O.generate_perm(Ar, Ac, "RS")
    prp, pcol, pval = O.apply_mat_perm(Ar, Ac, Av, perm, inv)
    if upper:
        row = np.repeat(np.arange(n), np.diff(prp))
        keep = pcol >= row
        trp = np.zeros(n + 1, np.int32)
        trp[1:] = np.cumsum(np.bincount(row[keep], minlength=n))
        tcol, tval = pcol[keep].copy(), pval[keep].copy()
    else:
        trp, tcol, tval = M.lower_triangle(prp, pcol, pval)
    b = np.random.default_rng(8).uniform(-1, 1, n)
    x = _run(trp, tcol, tval, b, SYNCFREE, upper=upper, perm_levels=lvl)
    assert normwise(x, O.sptrsv(trp, tcol, tval, b, lower=not upper, levels=lvl)) <= 1e-12
    np.testing.assert_array_equal(x, _run(trp, tcol, tval, b, MERGED, upper=upper, perm_levels=lvl))


def test_syncfree_config3_permuted_2048():
    """The 5-point 2048^2 lower triangle under the seed-3 random symmetric
    permutation, RS levels (15 levels of up to ~10^6 rows)."""
    from smaxkernels_b200 import matrices as M
    A = M.laplace2d_5pt(2048)
    Ar, Ac, Av, _ = M.random_symmetric_permutation(*A, seed=3)
    from smaxkernels_b200 import Interface
    n = len(Ar) - 1
    smax = Interface()
    perm = np.zeros(n, np.int32)
    inv = np.zeros(n, np.int32)
    smax.utils.generate_perm(n, Ar, Ac, perm, inv, "RS")
    prp = np.zeros(n + 1, np.int32)
    pcol = np.zeros(len(Ac), np.int32)
    pval = np.zeros(len(Ac))
    smax.utils.apply_mat_perm(n, Ar, Ac, Av, prp, pcol, pval, perm, inv)
    lvl = np.array([smax.get_level_ptr_at(i) for i in range(smax.get_n_levels() + 1)], np.int32)
    smax.close()
    lrp, lcol, lval = M.lower_triangle(prp, pcol, pval)
    b = M.uniform_vector(n, 3)
    x = _run(lrp, lcol, lval, b, SYNCFREE, perm_levels=lvl)
    assert normwise(x, O.sptrsv(lrp, lcol, lval, b, levels=lvl)) <= 1e-12
    np.testing.assert_array_equal(x, _run(lrp, lcol, lval, b, MERGED, perm_levels=lvl))


def test_syncfree_degenerate():
    # one row; a diagonal-only matrix (no dependencies at all)
    rp, col, val = np.array([0, 1], np.int32), np.array([0], np.int32), np.array([4.0])
    x = _run(rp, col, val, np.array([2.0]), SYNCFREE)
    assert x[0] == 0.5
    n = 1000
    rp = np.arange(n + 1, dtype=np.int32)
    col = np.arange(n, dtype=np.int32)
    val = np.random.default_rng(1).uniform(1, 2, n)
    b = np.random.default_rng(2).uniform(-1, 1, n)
    x = _run(rp, col, val, b, SYNCFREE)
    np.testing.assert_array_equal(x, _run(rp, col, val, b, MERGED))
    assert normwise(x, b / val) <= 1e-15


def test_syncfree_falls_back_when_a_row_reads_a_later_level():
    """Caller-given levels under which a row reads a row of a LATER level: the
    reference reads that row's initial x.  A sync-free row would wait for it
    forever, so the form does not apply and the merged solve runs instead.
    Rows 0..249 stand alone, row 250+i reads row i; the upper flag sweeps
    level 1 (rows 250..499) first."""
    n, h = 500, 250
    rng = np.random.default_rng(4)
    rp = np.concatenate([np.arange(h + 1), h + 2 * np.arange(1, h + 1)]).astype(np.int32)
    col = np.concatenate([np.arange(h), np.stack([np.arange(h), np.arange(h, n)], 1).ravel()]).astype(np.int32)
    val = np.concatenate([rng.uniform(2, 3, h), np.stack([np.full(h, -0.5), rng.uniform(2, 3, h)], 1).ravel()])
    lvl = np.array([0, h, n], np.int32)
    b = rng.uniform(-1, 1, n)
    x = _run(rp, col, val, b, SYNCFREE, upper=True, perm_levels=lvl)
    np.testing.assert_array_equal(x, _run(rp, col, val, b, MERGED, upper=True, perm_levels=lvl))
    assert normwise(x, O.sptrsv(rp, col, val, b, lower=False, levels=lvl)) <= 1e-12
    # rows 250.. read the initial (zero) x of rows 0..249
    np.testing.assert_allclose(x[h:], b[h:] / val[h + 1::2], rtol=1e-14)


def test_syncfree_in_place_falls_back():
    """B and X the same device array: the sync-free form marks X before it
    reads B, so an in-place solve runs merged; the result is the out-of-place one."""
    import torch
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    rp, col, val = rand_crs(4000, 6, 17, lower=True)
    n = len(rp) - 1
    b = np.random.default_rng(18).uniform(-1, 1, n)
    ref = _run(rp, col, val, b, SYNCFREE)
    smax = Interface()
    smax.register_kernel("t", KernelType.SPTRSV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("t")
    k.set_solve_mode(SYNCFREE)
    xb = torch.tensor(b, device="cuda")
    k.register_A(n, n, len(col), col.copy(), rp, val.copy())
    k.register_B(n, xb)
    k.register_C(n, xb)
    k.run()
    torch.cuda.synchronize()
    smax.close()
    np.testing.assert_array_equal(xb.cpu().numpy(), ref)


def test_syncfree_wait_timeout_is_an_error_and_recoverable():
    """The first row is made to wait on a value that is never written; the wait
    gives up after the spin limit, reports TIMEOUT, the other waits end on the
    abort flag, and the same kernel object solves correctly afterwards."""
    from smaxkernels_b200 import SmaxError, _lib
    rp, col, val = rand_crs(3000, 5, 141, lower=True)
    b = np.random.default_rng(142).uniform(-1, 1, 3000)
    smax, k, x = _solve(rp, col, val, b, SYNCFREE, spin=5, force_timeout=True)
    with pytest.raises(SmaxError) as e:
        k.run()
    assert e.value.code == _lib.ERR_TIMEOUT
    k._flag("test_force_timeout", 0)
    k.run()
    smax.close()
    assert normwise(x, O.sptrsv(rp, col, val, b)) <= 1e-12


def test_autotune_considers_syncfree():
    from smaxkernels_b200 import matrices as M
    # a size no other test tunes: choices are cached per matrix for the process
    lrp, lcol, lval = M.lower_triangle(*M.laplace2d_5pt(173))
    n = len(lrp) - 1
    b = M.uniform_vector(n, 3)
    smax, k, x = _solve(lrp, lcol, lval, b, 0)
    k.initialize()
    r = k.autotune()
    k.run()
    smax.close()
    assert r["n_candidates"] >= 9
    assert r["solve_mode"] in (2, 3, 4, 5)
    assert normwise(x, O.sptrsv(lrp, lcol, lval, b)) <= 1e-12


# ------------------------------------------------ SpTRSM, row-major blocks --
def _solve_m(rp, col, val, B, k_, mode, row_major=True, upper=False):
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    n = len(rp) - 1
    smax = Interface()
    smax.register_kernel("t", KernelType.SPTRSM, PlatformType.CUDA, IntType.INT32,
                         FloatType.FLOAT64 if val.dtype == np.float64 else FloatType.FLOAT32)
    k = smax.kernel("t")
    k.set_solve_mode(mode)
    if mode == MERGED:
        k.set_level_merge(0)
    if upper:
        k.set_mat_upper_triang(True)
    X = np.zeros(n * k_, val.dtype)
    k.register_A(n, n, len(col), col.copy(), rp, val.copy())
    k.register_B(n, k_, X)
    k.register_C(n, k_, np.ascontiguousarray(B, val.dtype))
    k.set_vec_row_major(row_major)
    k.run()
    smax.close()
    return X


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("k_", [2, 32, 40])
@pytest.mark.parametrize("upper", [False, True])
def test_syncfree_sptrsm_row_major(vt, k_, upper):
    """A warp per row, lanes over the right-hand sides (two passes for 40):
    the plain kernels' arithmetic, so the merged solve's bits."""
    rp, col, val = rand_crs(2500, 7, 81, vt=vt, lower=True)
    if upper:
        rp, col, val = _upper(rp, col, val)
    B = np.random.default_rng(82).uniform(-1, 1, 2500 * k_).astype(vt)
    X = _solve_m(rp, col, val, B, k_, SYNCFREE, upper=upper)
    assert normwise(X, O.sptrsm(rp, col, val, B, k_, row_major=True, lower=not upper)) <= tol(vt)
    np.testing.assert_array_equal(X, _solve_m(rp, col, val, B, k_, MERGED, upper=upper))


def test_syncfree_sptrsm_laplace_natural_default():
    """The natural 5-point 300^2 lower triangle with 32 right-hand sides
    (90,000 rows, 599 levels): the default scheme runs it sync-free."""
    from smaxkernels_b200 import matrices as M
    lrp, lcol, lval = M.lower_triangle(*M.laplace2d_5pt(300))
    n = len(lrp) - 1
    B = np.random.default_rng(3).uniform(-1, 1, n * 32)
    X = _solve_m(lrp, lcol, lval, B, 32, 0)
    assert normwise(X, O.sptrsm(lrp, lcol, lval, B, 32, row_major=True)) <= 1e-12
    np.testing.assert_array_equal(X, _solve_m(lrp, lcol, lval, B, 32, MERGED))


@pytest.mark.parametrize("k_", [5, 33])
@pytest.mark.parametrize("upper", [False, True])
def test_syncfree_sptrsm_column_major(k_, upper):
    """Column-major blocks (element (r, v) at r + v * n_rows, the reference's
    leading dimension): the same row kernel with strided vectors."""
    rp, col, val = rand_crs(1200, 6, 83, lower=True)
    if upper:
        rp, col, val = _upper(rp, col, val)
    B = np.random.default_rng(84).uniform(-1, 1, 1200 * k_)
    X = _solve_m(rp, col, val, B, k_, SYNCFREE, row_major=False, upper=upper)
    np.testing.assert_array_equal(X, _solve_m(rp, col, val, B, k_, MERGED, row_major=False, upper=upper))
    assert normwise(X, O.sptrsm(rp, col, val, B, k_, row_major=False, lower=not upper)) <= 1e-12


def test_syncfree_sptrsm_column_major_natural_default():
    """The natural 5-point 300^2 lower triangle, 8 column-major right-hand
    sides: the default scheme runs it sync-free."""
    from smaxkernels_b200 import matrices as M
    lrp, lcol, lval = M.lower_triangle(*M.laplace2d_5pt(300))
    n = len(lrp) - 1
    B = np.random.default_rng(5).uniform(-1, 1, n * 8)
    X = _solve_m(lrp, lcol, lval, B, 8, 0, row_major=False)
    assert normwise(X, O.sptrsm(lrp, lcol, lval, B, 8, row_major=False)) <= 1e-12
    np.testing.assert_array_equal(X, _solve_m(lrp, lcol, lval, B, 8, MERGED, row_major=False))
