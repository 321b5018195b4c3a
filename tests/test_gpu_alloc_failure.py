"""Device allocation failures: every allocation point of a kernel's first run,
made to fail one at a time, gives SMAX_ERR_OOM, and the SAME kernel object
then runs correctly once memory is available again.

The failure is injected on the host (smax_test_fail_device_alloc: the n-th
device allocation fails as an out-of-memory cudaMalloc would, without calling
it); no GPU is faulted.  The reference has no recovery to match: its CUDA
path prints a failed allocation and carries on (src/platforms/cuda/
cuda.cuh:23-44); here a failed allocation is an error status, the kernel
object keeps its registered operands, and the next run rebuilds whatever the
failed one left unfinished.
"""
import numpy as np
import pytest

from helpers import normwise, rand_crs
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
O = Oracle()


def _lib():
    from smaxkernels_b200 import _lib
    return _lib


def _count():
    return int(_lib().lib.smax_test_device_alloc_count())


def _arm(n):
    assert _lib().lib.smax_test_fail_device_alloc(n) == 0


def _spmv_case(scs=False):
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    rp, col, val = rand_crs(3000, 40, 91, empty_frac=0.1, long_rows=(1500,))
    n = len(rp) - 1
    x = np.random.default_rng(92).uniform(-1, 1, n)
    y_ref = O.spmv_crs(rp, col, val, x)
    smax = Interface()
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    if scs:
        s = O.scs(rp, col, val, 32, 64)
        vs = max(s["n_rows_padded"], n)
        xs = np.zeros(vs)
        xs[:n] = x
        y = np.zeros(vs)
        k.set_mat_scs(True)
        k.register_A(32, 64, s["n_rows"], s["n_rows_padded"], n, s["n_chunks"], s["n_elements"], s["nnz"],
                     s["chunk_ptr"], s["chunk_lengths"], s["col"], s["val"], s["perm"])
        k.register_B(vs, xs)
        k.register_C(vs, y)
        return smax, k, lambda: y[s["perm"][:n]], y_ref
    y = np.zeros(n)
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, x)
    k.register_C(n, y)
    return smax, k, lambda: y, y_ref


def _sptrsv_case():
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    rp, col, val = rand_crs(2500, 8, 93, lower=True)
    n = len(rp) - 1
    b = np.random.default_rng(94).uniform(-1, 1, n)
    x_ref = O.sptrsv(rp, col, val, b)
    smax = Interface()
    smax.register_kernel("k", KernelType.SPTRSV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    x = np.zeros(n)
    k.register_A(n, n, len(col), col.copy(), rp, val.copy())
    k.register_B(n, x)
    k.register_C(n, b)
    return smax, k, lambda: x, x_ref


def _spmm_case():
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    rp, col, val = rand_crs(2000, 20, 95)
    n, kk = len(rp) - 1, 16
    X = np.random.default_rng(96).uniform(-1, 1, n * kk)
    Y_ref = O.spmm(rp, col, val, X, kk, row_major=True)
    smax = Interface()
    smax.register_kernel("k", KernelType.SPMM, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    Y = np.zeros(n * kk)
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, kk, X)
    k.register_C(n, kk, Y)
    k.set_vec_row_major(True)
    return smax, k, lambda: Y, Y_ref


def _spgemm_case():
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    A = rand_crs(1500, 12, 97, long_rows=(700,))
    orp, ocol, oval = O.spgemm(*A, *A, 1500)
    smax = Interface()
    smax.register_kernel("k", KernelType.SPGEMM, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    rp, col, val = A
    k.register_A(1500, 1500, len(col), col, rp, val)
    k.register_B(1500, 1500, len(col), col, rp, val)
    k.register_C()

    def result():
        _, _, _, crp, ccol, cval = k.result()
        np.testing.assert_array_equal(crp, orp)
        np.testing.assert_array_equal(ccol, ocol)
        return cval
    return smax, k, result, oval


CASES = {"spmv_crs": _spmv_case, "spmv_scs": lambda: _spmv_case(scs=True), "sptrsv": _sptrsv_case,
         "spmm": _spmm_case, "spgemm": _spgemm_case}


@pytest.mark.parametrize("name", sorted(CASES))
def test_every_allocation_point_fails_cleanly_and_the_kernel_recovers(name):
    from smaxkernels_b200 import SmaxError
    _arm(0)
    # how many device allocations the first run makes
    smax, k, _, _ = CASES[name]()
    c0 = _count()
    k.run()
    n_allocs = _count() - c0
    smax.close()
    assert n_allocs >= 1, "the first run allocated nothing on the device"
    for nth in range(1, n_allocs + 1):
        smax, k, result, ref = CASES[name]()
        _arm(nth)
        with pytest.raises(SmaxError) as e:
            k.run()
        assert e.value.code == _lib().ERR_OOM, (nth, str(e.value))
        assert b"injected" in _lib().lib.smax_last_error()
        _arm(0)
        k.run()  # the same kernel object, memory available again
        assert normwise(result(), ref) <= 1e-12, (name, nth)
        smax.close()
    _arm(0)


def test_injection_disarms_itself_and_can_be_cleared():
    from smaxkernels_b200 import SmaxError
    smax, k, result, ref = _spmv_case()
    _arm(1)
    with pytest.raises(SmaxError):
        k.run()
    k.run()  # disarmed after firing once
    assert normwise(result(), ref) <= 1e-12
    smax.close()
    _arm(1)
    _arm(0)  # cleared before any allocation
    smax, k, result, ref = _spmv_case()
    k.run()
    assert normwise(result(), ref) <= 1e-12
    smax.close()
    assert _lib().lib.smax_test_fail_device_alloc(-1) == _lib().ERR_BAD_ARG
