"""Batched SpTRSV (persistent kernel with a device work queue), the grid-wide
persistent solve, and the bounded barrier of the latter (timeout knob)."""
import numpy as np
import pytest

from helpers import normwise, rand_crs, tol
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
O = Oracle()


def _lower_laplace(side, dtype=np.float64):
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace2d_5pt(side, dtype=dtype)
    return M.lower_triangle(rp, col, val)


def _batch_mats(vt, sides=(3, 17, 40, 9, 64, 1), randoms=4):
    mats = [_lower_laplace(s, vt) for s in sides]
    for i in range(randoms):
        mats.append(rand_crs(300 + 200 * i, 6, 120 + i, vt=vt, lower=True))
    return mats


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("mode", [3, 2, 1])
def test_batch_vs_oracle(vt, mode):
    import torch
    from smaxkernels_b200.interface import FloatType, TriangularBatch
    mats = _batch_mats(vt)
    tdt = torch.float64 if vt == np.float64 else torch.float32
    tb = TriangularBatch(mats, FloatType.FLOAT64 if vt == np.float64 else FloatType.FLOAT32)
    n, total_levels, max_levels = tb.info()
    assert n == sum(len(m[0]) - 1 for m in mats)
    rng = np.random.default_rng(7)
    b = rng.uniform(-1, 1, n).astype(vt)
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros(n, dtype=tdt, device="cuda")
    for rep in range(2):  # the graph is captured on the first call and replayed
        xd.zero_()
        torch.cuda.synchronize()
        tb.solve(bd, xd, mode)
        torch.cuda.synchronize()
        x = xd.cpu().numpy()
        for m, (rp, col, val) in enumerate(mats):
            a, e = tb.row_offset(m), tb.row_offset(m + 1)
            x_ref = O.sptrsv(rp, col, val, b[a:e])
            assert normwise(x[a:e], x_ref) <= tol(vt), (m, rep)
    tb.close()


def test_batch_does_not_modify_caller_arrays():
    from smaxkernels_b200.interface import TriangularBatch
    rp, col, val = rand_crs(200, 5, 3, lower=True)
    # move each diagonal to the front so a peel would have to change the arrays
    col2, val2 = col.copy(), val.copy()
    for r in range(200):
        s, e = rp[r], rp[r + 1]
        col2[s:e] = np.roll(col[s:e], 1)
        val2[s:e] = np.roll(val[s:e], 1)
    c0, v0 = col2.copy(), val2.copy()
    tb = TriangularBatch([(rp, col2, val2)])
    tb.close()
    np.testing.assert_array_equal(col2, c0)
    np.testing.assert_array_equal(val2, v0)


@pytest.mark.slow
def test_batch_64_laplacians():
    """The batch of the triangular-solve configuration: 64 lower triangles of
    5-point Laplacians with sides 100 + round(600*i/63)."""
    import torch
    from smaxkernels_b200.interface import TriangularBatch
    sides = [100 + int(round(600 * i / 63)) for i in range(64)]
    mats = [_lower_laplace(s) for s in sides]
    tb = TriangularBatch(mats)
    n, total_levels, max_levels = tb.info()
    assert n == sum(s * s for s in sides)
    assert max_levels == 2 * 700 - 1 and total_levels == sum(2 * s - 1 for s in sides)
    b = np.random.default_rng(3).uniform(-1, 1, n)
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    tb.solve(bd, xd, 3)
    torch.cuda.synchronize()
    x = xd.cpu().numpy()
    for m in (0, 31, 63):
        rp, col, val = mats[m]
        a, e = tb.row_offset(m), tb.row_offset(m + 1)
        assert normwise(x[a:e], O.sptrsv(rp, col, val, b[a:e])) <= 1e-12
    tb.close()


# ------------------------------------------------------ grid persistent ----
def _run_single(rp, col, val, b, mode, upper=False, spin=None, force_timeout=False):
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    n = len(rp) - 1
    smax = Interface()
    smax.register_kernel("t", KernelType.SPTRSV, PlatformType.CUDA, IntType.INT32,
                         FloatType.FLOAT64 if val.dtype == np.float64 else FloatType.FLOAT32)
    k = smax.kernel("t")
    k.set_solve_mode(mode)
    if upper:
        k.set_mat_upper_triang(True)
    if spin:
        k.set_spin_limit(spin)
    if force_timeout:
        k._flag("test_force_timeout", 1)
    x = np.zeros(n, val.dtype)
    k.register_A(n, n, len(col), col.copy(), rp, val.copy())
    k.register_B(n, x)
    k.register_C(n, b)
    return smax, k, x


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("upper", [False, True])
def test_persistent_solve_vs_oracle(vt, upper):
    rp, col, val = rand_crs(5000, 7, 131, vt=vt, lower=True)
    if upper:
        import scipy.sparse as sp
        U = sp.csr_matrix((val, col, rp), shape=(5000, 5000)).T.tocsr()
        U.sort_indices()
        rp, col, val = U.indptr.astype(np.int32), U.indices.astype(np.int32), U.data.astype(vt)
    b = np.random.default_rng(132).uniform(-1, 1, 5000).astype(vt)
    smax, k, x = _run_single(rp, col, val, b, mode=4, upper=upper)
    k.run()
    smax.close()
    assert normwise(x, O.sptrsv(rp, col, val, b, lower=not upper)) <= tol(vt)


def test_persistent_barrier_timeout_is_an_error_and_recoverable():
    """The grid barrier is made to wait for an arrival that never comes; it
    gives up after the spin limit, reports TIMEOUT, and the same kernel object
    solves correctly once the knob is cleared."""
    from smaxkernels_b200 import SmaxError, _lib
    rp, col, val = rand_crs(3000, 5, 141, lower=True)
    b = np.random.default_rng(142).uniform(-1, 1, 3000)
    smax, k, x = _run_single(rp, col, val, b, mode=4, spin=5, force_timeout=True)
    with pytest.raises(SmaxError) as e:
        k.run()
    assert e.value.code == _lib.ERR_TIMEOUT
    k._flag("test_force_timeout", 0)
    k.run()
    smax.close()
    assert normwise(x, O.sptrsv(rp, col, val, b)) <= 1e-12
