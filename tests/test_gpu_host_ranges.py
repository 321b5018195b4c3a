"""Host-pointer mode: finalize() downloads exactly what apply() wrote (entries
of a larger output array outside the written range keep the caller's values,
several offsets before one finalize), and the pipelined CRS SpMV (row blocks
whose y is downloaded while later blocks compute) gives the oracle's result."""
import numpy as np
import pytest

from helpers import normwise, rand_crs, tol
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
O = Oracle()


def _spmv_kernel(vt, pipeline=None):
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    smax = Interface()
    smax.register_kernel("s", KernelType.SPMV, PlatformType.CUDA, IntType.INT32,
                         FloatType.FLOAT64 if vt == np.float64 else FloatType.FLOAT32)
    k = smax.kernel("s")
    if pipeline is not None:
        k._flag("spmv_pipeline", pipeline)
    return smax, k


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("pipeline", [0, 4, 7, 16, None])
def test_pipelined_spmv_matches_oracle(vt, pipeline):
    """Geometric row blocks (None: the default count); x changes between
    runs, which upload it without waiting before the apply."""
    n = 300_000
    rp, col, val = rand_crs(n, 12, 77, vt=vt, empty_frac=0.05, long_rows=(40000, 9000, 5000))
    rng = np.random.default_rng(78)
    x = rng.uniform(-1, 1, n).astype(vt)
    smax, k = _spmv_kernel(vt, pipeline)
    y = np.zeros(n, vt)
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, x)
    k.register_C(n, y)
    for _ in range(3):  # plans built on the first apply, reused after
        x[:] = rng.uniform(-1, 1, n).astype(vt)
        y_ref = O.spmv_crs(rp, col, val, x)
        y[:] = 7.0
        k.run()
        assert normwise(y, y_ref) <= tol(vt)
    smax.close()


def test_finalize_leaves_untouched_entries_alone():
    n = 5000
    rp, col, val = rand_crs(n, 9, 80)
    x = np.random.default_rng(81).uniform(-1, 1, n)
    y_ref = O.spmv_crs(rp, col, val, x)
    smax, k = _spmv_kernel(np.float64)
    big = np.full(3 * n + 11, -3.25)
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, x)
    k.register_C(len(big), big)
    k.initialize()
    k.apply(0, 0, n + 5)           # y into big[n+5 : 2n+5]
    k.apply(0, 0, 2 * n + 11)      # and into big[2n+11 : 3n+11]
    k.finalize()
    np.testing.assert_array_equal(big[: n + 5], -3.25)
    assert normwise(big[n + 5: 2 * n + 5], y_ref) <= 1e-12
    np.testing.assert_array_equal(big[2 * n + 5: 2 * n + 11], -3.25)
    assert normwise(big[2 * n + 11:], y_ref) <= 1e-12
    # a finalize without apply copies nothing
    big2 = big.copy()
    k.finalize()
    np.testing.assert_array_equal(big, big2)
    smax.close()


def test_repeated_applies_then_one_finalize():
    n = 400_000  # pipelined
    rp, col, val = rand_crs(n, 6, 82)
    x = np.random.default_rng(83).uniform(-1, 1, n)
    smax, k = _spmv_kernel(np.float64)
    y = np.zeros(n)
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, x)
    k.register_C(n, y)
    k.initialize()
    for _ in range(50):
        k.apply()
    k.finalize()
    assert normwise(y, O.spmv_crs(rp, col, val, x)) <= 1e-12
    smax.close()


def test_sptrsv_host_mode_downloads_the_solution_only():
    n = 3000
    rp, col, val = rand_crs(n, 5, 84, lower=True)
    b = np.random.default_rng(85).uniform(-1, 1, n)
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    smax = Interface()
    smax.register_kernel("t", KernelType.SPTRSV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("t")
    xbig = np.full(n + 9, 1.5)
    col2, val2 = col.copy(), val.copy()
    k.register_A(n, n, len(col), col2, rp, val2)
    k.register_B(len(xbig), xbig)
    k.register_C(n, b)
    k.initialize()
    k.apply(0, 9, 0)
    k.finalize()
    np.testing.assert_array_equal(xbig[:9], 1.5)
    assert normwise(xbig[9:], O.sptrsv(rp, col, val, b)) <= 1e-12
    smax.close()
