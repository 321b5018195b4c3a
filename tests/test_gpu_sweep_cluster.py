"""Level-pack solves whose runs have levels wider than 1024 rows, with
cluster runs enabled: these run on a thread-block cluster (8 CTAs, solutions
shared through distributed shared memory).  Checked against the oracle, lower and upper, FP64 and FP32, with
long-distance couplings that must be read from global memory, and through
the adjoint (the reversed plan)."""
import numpy as np
import pytest
import scipy.sparse as sp

from helpers import normwise, tol
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
O = Oracle()


def _kernel(vt, upper=False, mode=0):
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    smax = Interface()
    smax.register_kernel("t", KernelType.SPTRSV, PlatformType.CUDA, IntType.INT32,
                         FloatType.FLOAT64 if vt == np.float64 else FloatType.FLOAT32)
    k = smax.kernel("t")
    if upper:
        k.set_mat_upper_triang(True)
    k.set_solve_mode(mode)
    k.set_sweep_cluster(True)
    return smax, k


def _solve(rp, col, val, b, upper=False, mode=0):
    n = len(rp) - 1
    smax, k = _kernel(val.dtype.type, upper, mode)
    x = np.zeros(n, val.dtype)
    col, val = col.copy(), val.copy()
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, x)
    k.register_C(n, b)
    k.run()
    return smax, k, x, col, val


def _laplace_lower(side, vt):
    from smaxkernels_b200 import matrices as M
    return M.lower_triangle(*M.laplace2d_5pt(side, dtype=vt))


def _csr(rp, col, val, n):
    A = sp.csr_matrix((val, col, rp), shape=(n, n))
    A.sort_indices()
    return A


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("side", [1500, 2200])
@pytest.mark.parametrize("mode", [0, 2])
def test_wide_levels_lower(vt, side, mode):
    rp, col, val = _laplace_lower(side, vt)
    b = np.random.default_rng(side).uniform(-1, 1, len(rp) - 1).astype(vt)
    smax, k, x, _, _ = _solve(rp, col, val, b, mode=mode)
    assert normwise(x, O.sptrsv(rp, col, val, b)) <= tol(vt)
    smax.close()


@pytest.mark.parametrize("vt", [np.float64, np.float32])
def test_wide_levels_upper(vt):
    rp, col, val = _laplace_lower(1300, vt)
    n = len(rp) - 1
    U = _csr(rp, col, val, n).T.tocsr()
    U.sort_indices()
    urp, ucol, uval = U.indptr.astype(np.int32), U.indices.astype(np.int32), U.data.astype(vt)
    b = np.random.default_rng(5).uniform(-1, 1, n).astype(vt)
    smax, k, x, _, _ = _solve(urp, ucol, uval, b, upper=True)
    assert normwise(x, O.sptrsv(urp, ucol, uval, b, lower=False)) <= tol(vt)
    smax.close()


def test_wide_levels_with_long_distance_couplings():
    """Extra entries (r, r - 9000): some solutions are older than the ring or
    were solved by another CTA of the cluster, and come from global memory."""
    rp, col, val = _laplace_lower(1400, np.float64)
    n = len(rp) - 1
    A = _csr(rp, col, val, n).tolil()
    rng = np.random.default_rng(11)
    for r in range(9000, n, 7):
        A[r, r - 9000] = rng.uniform(-0.2, 0.2)
    A = A.tocsr()
    A.sort_indices()
    rp2, col2, val2 = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data
    b = rng.uniform(-1, 1, n)
    smax, k, x, _, _ = _solve(rp2, col2, val2, b)
    assert normwise(x, O.sptrsv(rp2, col2, val2, b)) <= 1e-12
    smax.close()


def test_wide_levels_adjoint():
    rp, col, val = _laplace_lower(1500, np.float64)
    n = len(rp) - 1
    b = np.random.default_rng(12).uniform(-1, 1, n)
    g = np.random.default_rng(13).uniform(-1, 1, n)
    smax, k, x, pcol, pval = _solve(rp, col, val, b)
    lam = np.zeros(n)
    dval = np.zeros(len(col))
    k.adjoint(g, lam, dval)
    lam_ref, dval_ref = O.sptrsv_adjoint(rp, pcol, pval, x, g)
    assert normwise(lam, lam_ref) <= 1e-12
    assert normwise(dval, dval_ref) <= 1e-12
    smax.close()

