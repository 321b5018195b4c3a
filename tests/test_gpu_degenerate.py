"""Degenerate inputs through every kernel type: matrices with no rows, with
rows but no entries, and 1 x 1 -- each must run and give the oracle's (empty
or trivial) result, never an error or a device fault."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _k(ktype, vt=np.float64):
    from smaxkernels_b200 import FloatType, Interface, IntType, PlatformType
    smax = Interface()
    smax.register_kernel("k", ktype, PlatformType.CUDA, IntType.INT32,
                         FloatType.FLOAT64 if vt == np.float64 else FloatType.FLOAT32)
    return smax, smax.kernel("k")


E_I = np.zeros(0, np.int32)
E_V = np.zeros(0)


@pytest.mark.parametrize("variant", [1, 2])
def test_spmv_no_rows(variant):
    from smaxkernels_b200 import KernelType
    smax, k = _k(KernelType.SPMV)
    k.set_spmv_variant(variant)
    k.register_A(0, 0, 0, E_I, np.zeros(1, np.int32), E_V)
    k.register_B(0, np.zeros(0))
    k.register_C(0, np.zeros(0))
    k.run()
    smax.close()


def test_spmv_one_by_one_and_adjoint():
    from smaxkernels_b200 import KernelType
    smax, k = _k(KernelType.SPMV)
    x, y = np.array([3.0]), np.zeros(1)
    k.register_A(1, 1, 1, np.array([0], np.int32), np.array([0, 1], np.int32), np.array([2.5]))
    k.register_B(1, x)
    k.register_C(1, y)
    k.run()
    assert y[0] == 7.5
    dx, dval = np.zeros(1), np.zeros(1)
    k.adjoint(np.array([2.0]), dx, dval)
    assert dx[0] == 5.0 and dval[0] == 6.0
    smax.close()


def test_spmv_rows_without_entries_adjoint():
    from smaxkernels_b200 import KernelType
    smax, k = _k(KernelType.SPMV)
    n = 5
    x, y = np.ones(n), np.full(n, 9.0)
    k.register_A(n, n, 0, E_I, np.zeros(n + 1, np.int32), E_V)
    k.register_B(n, x)
    k.register_C(n, y)
    k.run()
    np.testing.assert_array_equal(y, 0.0)
    dx = np.full(n, 4.0)
    k.adjoint(np.ones(n), dx, None)
    np.testing.assert_array_equal(dx, 0.0)
    smax.close()


@pytest.mark.parametrize("mode", [0, 1, 2, 4])
def test_sptrsv_no_rows_and_one_row(mode):
    from smaxkernels_b200 import KernelType
    smax, k = _k(KernelType.SPTRSV)
    k.set_solve_mode(mode)
    k.register_A(0, 0, 0, E_I, np.zeros(1, np.int32), E_V)
    k.register_B(0, np.zeros(0))
    k.register_C(0, np.zeros(0))
    k.run()
    smax.close()
    smax, k = _k(KernelType.SPTRSV)
    k.set_solve_mode(mode)
    x = np.zeros(1)
    k.register_A(1, 1, 1, np.array([0], np.int32), np.array([0, 1], np.int32), np.array([4.0]))
    k.register_B(1, x)
    k.register_C(1, np.array([2.0]))
    k.run()
    assert x[0] == 0.5
    smax.close()


def test_spmm_no_rows():
    from smaxkernels_b200 import KernelType
    smax, k = _k(KernelType.SPMM)
    k.set_vec_row_major(True)
    k.register_A(0, 0, 0, E_I, np.zeros(1, np.int32), E_V)
    k.register_B(0, 4, np.zeros(0))
    k.register_C(0, 4, np.zeros(0))
    k.run()
    smax.close()


def test_spgemm_without_entries():
    from smaxkernels_b200 import KernelType
    smax, k = _k(KernelType.SPGEMM)
    rp = np.zeros(11, np.int32)
    k.register_A(10, 10, 0, E_I, rp, E_V)
    k.register_B(10, 10, 0, E_I, rp, E_V)
    k.register_C()
    k.run()
    n_rows, n_cols, nnz, crp, ccol, cval = k.result()
    assert (n_rows, n_cols, nnz) == (10, 10, 0)
    np.testing.assert_array_equal(crp, 0)
    smax.close()


def test_scs_conversion_of_rows_without_entries():
    from smaxkernels_b200 import Interface, KernelType
    smax = Interface()
    s = smax.utils.convert_crs_to_scs(6, 6, 0, E_I, np.zeros(7, np.int32), E_V, 4, 1)
    assert s["n_elements"] == 0 and s["n_chunks"] == 2
    smax.close()
    smax, k = _k(KernelType.SPMV)
    k.set_mat_scs(True)
    y = np.full(s["n_rows_padded"], 5.0)
    k.register_A(4, 1, s["n_rows"], s["n_rows_padded"], 6, s["n_chunks"], s["n_elements"], s["nnz"],
                 s["chunk_ptr"], s["chunk_lengths"], s["col"], s["val"], s["perm"])
    k.register_B(s["n_rows_padded"], np.ones(s["n_rows_padded"]))
    k.register_C(s["n_rows_padded"], y)
    k.run()
    np.testing.assert_array_equal(y, 0.0)
    smax.close()
