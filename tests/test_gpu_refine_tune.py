"""FP32 SpTRSV with FP64-residual refinement against the FP64 oracle, and the
autotuners (kernel launch variants with the per-matrix cache; storage format
of an SpMV matrix)."""
import numpy as np
import pytest

from helpers import normwise, rand_crs
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
O = Oracle()


def _tri_kernel(rp, col, val, b, upper=False):
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    n = len(rp) - 1
    smax = Interface()
    smax.register_kernel("t", KernelType.SPTRSV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("t")
    if upper:
        k.set_mat_upper_triang(True)
    x = np.zeros(n)
    col, val = col.copy(), val.copy()
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, x)
    k.register_C(n, b)
    return smax, k, x


def _lower_laplace(side):
    from smaxkernels_b200 import matrices as M
    return M.lower_triangle(*M.laplace2d_5pt(side))


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_refine_two_steps_reaches_fp64(mode):
    rp, col, val = _lower_laplace(256)
    n = len(rp) - 1
    b = np.random.default_rng(3).uniform(-1, 1, n)
    smax, k, x = _tri_kernel(rp, col, val, b)
    k.set_solve_mode(mode)
    k.set_refine(2)
    for _ in range(2):  # second run replays the captured sequence
        x[:] = 0
        k.run()
        assert normwise(x, O.sptrsv(rp, col, val, b)) <= 1e-12
    steps, rel = k.refine_stats()
    assert steps == 2 and 0 <= rel < 1e-12
    smax.close()


def test_refine_one_correction_and_off():
    rp, col, val = _lower_laplace(128)
    n = len(rp) - 1
    b = np.random.default_rng(4).uniform(-1, 1, n)
    smax, k, x = _tri_kernel(rp, col, val, b)
    k.set_refine(1)
    k.run()
    e1 = normwise(x, O.sptrsv(rp, col, val, b))
    smax.close()
    # zero corrections is "refinement off": the plain FP64 solve
    smax, k, x = _tri_kernel(rp, col, val, b)
    k.set_refine(0)
    k.run()
    assert normwise(x, O.sptrsv(rp, col, val, b)) <= 1e-14
    smax.close()
    assert e1 <= 1e-9  # one correction: ~u32^2 cond


@pytest.mark.parametrize("upper", [False, True])
def test_refine_tolerance_stops_early_random(upper):
    n = 6000
    rp, col, val = rand_crs(n, 7, 500, lower=True)
    if upper:
        import scipy.sparse as sp
        U = sp.csr_matrix((val, col, rp), shape=(n, n)).T.tocsr()
        U.sort_indices()
        rp, col, val = U.indptr.astype(np.int32), U.indices.astype(np.int32), U.data
    # a diagonally dominant triangle: well conditioned
    rows = np.repeat(np.arange(n), np.diff(rp))
    val = np.where(col == rows, 8.0 + np.abs(val), val)
    b = np.random.default_rng(501).uniform(-1, 1, n)
    smax, k, x = _tri_kernel(rp, col, val, b, upper)
    k.set_refine(10, 14)
    k.run()
    steps, rel = k.refine_stats()
    assert 1 <= steps < 10 and rel <= 1e-14
    assert normwise(x, O.sptrsv(rp, col, val, b, lower=not upper)) <= 1e-12
    smax.close()


def test_refine_rejects_float32_kernel():
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType, SmaxError, _lib
    smax = Interface()
    smax.register_kernel("t", KernelType.SPTRSV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT32)
    with pytest.raises(SmaxError) as e:
        smax.kernel("t").set_refine(2)
    assert e.value.code == _lib.ERR_UNSUPPORTED_TYPE
    smax.close()


def test_refine_follows_value_updates():
    rp, col, val = _lower_laplace(100)
    n = len(rp) - 1
    b = np.random.default_rng(5).uniform(-1, 1, n)
    smax, k, x = _tri_kernel(rp, col, val, b)
    k.set_refine(2)
    k.run()
    # after run the registered arrays hold the diagonal-last order
    col2, val2 = k._keep["A"][0], k._keep["A"][2] * 1.25
    k.update_A_values(val2)
    k.apply()
    k.finalize()
    assert normwise(x, O.sptrsv(rp, col2, val2, b)) <= 1e-12
    smax.close()


# ------------------------------------------------------------- autotuner ----
def test_autotune_spmv_and_cache():
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.lognormal_random(1 << 16, seed=11)
    n = len(rp) - 1
    x = np.random.default_rng(12).uniform(-1, 1, n)
    choices = []
    for rep in range(2):
        smax = Interface()
        smax.register_kernel("s", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
        k = smax.kernel("s")
        y = np.zeros(n)
        k.register_A(n, n, len(col), col, rp, val)
        k.register_B(n, x)
        k.register_C(n, y)
        k.initialize()
        t = k.autotune()
        choices.append(t)
        assert t["spmv_variant"] in (1, 2) and t["seconds"] > 0
        k.apply()
        k.finalize()
        assert normwise(y, O.spmv_crs(rp, col, val, x)) <= 1e-12
        smax.close()
    assert choices[0]["from_cache"] == 0 and choices[0]["n_candidates"] == 2
    assert choices[1]["from_cache"] == 1 and choices[1]["spmv_variant"] == choices[0]["spmv_variant"]


def test_autotune_sptrsv():
    rp, col, val = _lower_laplace(200)
    n = len(rp) - 1
    b = np.random.default_rng(6).uniform(-1, 1, n)
    smax, k, x = _tri_kernel(rp, col, val, b)
    k.initialize()
    t = k.autotune()
    assert t["solve_mode"] in (3, 4) and t["n_candidates"] >= 5
    k.apply()
    k.finalize()
    assert normwise(x, O.sptrsv(rp, col, val, b)) <= 1e-12
    smax.close()


def test_tune_spmv_format():
    from smaxkernels_b200 import Interface
    rp, col, val = rand_crs(20000, 30, 13, n_cols=20000)
    smax = Interface()
    c = smax.utils.tune_spmv_format(20000, 20000, len(col), col, rp, val)
    smax.close()
    assert c["format"] in (0, 1, 2) and c["n_candidates"] >= 12
    assert 0 < c["seconds"] <= c["crs_seconds"]
    if c["format"] == 1:
        assert c["C"] in (8, 16, 32, 64)
