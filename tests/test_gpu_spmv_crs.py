"""Parity of the CUDA CRS SpMV with the oracle (and the reference's golden
vectors), through the C ABI via the Python mirror of SMAX::Interface."""
import numpy as np
import pytest

import golden_cases as G
from helpers import gpu_spmv, normwise, rand_crs, tol
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
O = Oracle()


def test_golden_spmv_test():
    c = G.spmv_case()
    y = gpu_spmv(c["row_ptr"], c["col"], c["val"], c["x"])
    assert G.almost_equal(y, c["y"], np.float64)


@pytest.mark.parametrize("variant", [1, 2])
@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("case", ["small", "empty_rows", "long_rows", "single_row", "ragged", "mostly_empty"])
def test_random_vs_oracle(vt, case, variant):
    kw = dict(small=dict(n=257, maxlen=9), empty_rows=dict(n=3001, maxlen=40, empty_frac=0.5),
              long_rows=dict(n=5000, maxlen=20, long_rows=(1025, 2049, 4097, 4999)),
              single_row=dict(n=1, maxlen=1, n_cols=7000, long_rows=(6000,)),
              ragged=dict(n=20011, maxlen=300), mostly_empty=dict(n=4099, maxlen=3, empty_frac=0.95))[case]
    n_cols = kw.pop("n_cols", None)
    rp, col, val = rand_crs(seed=11, vt=vt, n_cols=n_cols, **kw)
    x = np.random.default_rng(12).uniform(-1, 1, n_cols or len(rp) - 1).astype(vt)
    y = gpu_spmv(rp, col, val, x, variant=variant)
    y_ref = O.spmv_crs(rp, col, val, x)  # reference arithmetic in VT
    assert normwise(y, y_ref) <= tol(vt)
    y64 = O.spmv_crs(rp, col, val.astype(np.float64), x.astype(np.float64))
    assert normwise(y, y64) <= tol(vt)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("longest", [32, 33])
def test_stream_short_row_bound(vt, longest):
    """Rows of at most 32 entries run the one-launch mode (each slice sums the
    head of its first row); one row of 33 switches to slice carries."""
    rp, col, val = rand_crs(50000, 32, seed=41, vt=vt, empty_frac=0.1, long_rows=(longest,) * 3)
    assert np.diff(rp).max() == longest
    x = np.random.default_rng(42).uniform(-1, 1, len(rp) - 1).astype(vt)
    y = gpu_spmv(rp, col, val, x, variant=1)
    assert normwise(y, O.spmv_crs(rp, col, val, x)) <= tol(vt)
    y64 = O.spmv_crs(rp, col, val.astype(np.float64), x.astype(np.float64))
    assert normwise(y, y64) <= tol(vt)


@pytest.mark.parametrize("variant", [1, 2])
def test_all_rows_empty(variant):
    n = 1000
    rp = np.zeros(n + 1, np.int32)
    y = gpu_spmv(rp, np.zeros(0, np.int32), np.zeros(0), np.ones(n), variant=variant)
    assert np.all(y == 0)


def test_config0_laplace64():
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace3d_7pt(64)
    x = M.uniform_vector(len(rp) - 1, 0)
    y = gpu_spmv(rp, col, val, x)
    assert normwise(y, O.spmv_crs(rp, col, val, x)) <= 1e-12


@pytest.mark.slow
@pytest.mark.parametrize("variant", [1, 2])
@pytest.mark.parametrize("vt", [np.float64, np.float32])
def test_config1_lognormal_full_size(vt, variant):
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.lognormal_random(1 << 22, dtype=vt)
    x = M.uniform_vector(len(rp) - 1, 1, dtype=vt)
    y = gpu_spmv(rp, col, val, x, variant=variant)
    assert normwise(y, O.spmv_crs(rp, col, val, x)) <= tol(vt)
    y64 = O.spmv_crs(rp, col, val.astype(np.float64), x.astype(np.float64))
    assert normwise(y, y64) <= tol(vt)


def test_offsets_and_repeated_runs():
    """x/y offsets (src/kernel.hpp:99-111) and reuse of the resident matrix."""
    from smaxkernels_b200 import FloatType, Interface, KernelType, PlatformType, IntType
    rp, col, val = rand_crs(2000, 30, 5)
    n = 2000
    X = np.random.default_rng(1).uniform(-1, 1, 2 * n)
    Y = np.zeros(2 * n)
    smax = Interface()
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(2 * n, X)
    k.register_C(2 * n, Y)
    k.run(0, n, 0)
    k.run(0, 0, n)
    assert normwise(Y[:n], O.spmv_crs(rp, col, val, X[n:])) <= 1e-12
    assert normwise(Y[n:], O.spmv_crs(rp, col, val, X[:n])) <= 1e-12
    assert k.timer("apply") > 0
    import io
    buf = io.StringIO()
    smax.utils.print_timers(file=buf)
    text = buf.getvalue()
    assert "Total time in 'k'" in text and "Apply time" in text
    smax.close()


def test_device_pointers_torch():
    import torch
    from smaxkernels_b200 import FloatType, Interface, KernelType, PlatformType, IntType
    rp, col, val = rand_crs(4000, 50, 6)
    x = torch.rand(4000, dtype=torch.float64, device="cuda")
    y = torch.zeros(4000, dtype=torch.float64, device="cuda")
    smax = Interface()
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    k.register_A(4000, 4000, len(col), col, rp, val)
    k.register_B(4000, x)
    k.register_C(4000, y)
    k.run()
    assert normwise(y.cpu().numpy(), O.spmv_crs(rp, col, val, x.cpu().numpy())) <= 1e-12
    smax.close()


@pytest.mark.parametrize("poison", ["col_oob", "col_negative", "row_ptr_decreasing", "row_ptr_end"])
def test_malformed_matrix_is_an_error_status(poison):
    """Malformed CRS input is rejected by the upload-time validation pass with
    an error status (the reference aborts in debug mode,
    src/kernels/kernels_common.hpp:21-28); no kernel reads out of bounds."""
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType, SmaxError
    from smaxkernels_b200 import _lib
    rp, col, val = rand_crs(300, 10, 3)
    rp = rp.copy()
    col = col.copy()
    expect = _lib.ERR_COL_OOB
    if poison == "col_oob":
        col[len(col) // 2] = 300
    elif poison == "col_negative":
        col[0] = -1
    elif poison == "row_ptr_decreasing":
        rp[100], rp[101] = rp[101] + 1, rp[100]
        expect = _lib.ERR_BAD_ARG
    else:
        rp[-1] = len(col) - 1
        expect = _lib.ERR_BAD_ARG
    smax = Interface()
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    k.register_A(300, 300, len(col), col, rp, val)
    k.register_B(300, np.ones(300))
    k.register_C(300, np.zeros(300))
    with pytest.raises(SmaxError) as e:
        k.run()
    assert e.value.code == expect
    # the kernel object stays usable after the error
    rp2, col2, val2 = rand_crs(300, 10, 3)
    x = np.ones(300)
    y = np.zeros(300)
    k.register_A(300, 300, len(col2), col2, rp2, val2)
    k.register_B(300, x)
    k.register_C(300, y)
    k.run()
    assert normwise(y, O.spmv_crs(rp2, col2, val2, x)) <= 1e-12
    smax.close()


def test_operand_too_small_is_rejected():
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType, SmaxError
    rp, col, val = rand_crs(300, 10, 3)
    smax = Interface()
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    k.register_A(300, 300, len(col), col, rp, val)
    k.register_B(300, np.ones(300))
    k.register_C(299, np.zeros(299))
    with pytest.raises(SmaxError):
        k.run()
    smax.close()


def test_timers_off_records_no_apply_time():
    """SMAX_FLAG_TIMERS = 0: applies record no CUDA events and the apply
    timer stays 0; the results are unchanged.  Switched back on, the timer
    counts again."""
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    rp, col, val = rand_crs(3000, 20, 6)
    n = 3000
    x = np.random.default_rng(2).uniform(-1, 1, n)
    y = np.zeros(n)
    smax = Interface()
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    k.set_timers(False)
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, x)
    k.register_C(n, y)
    for _ in range(3):
        k.run()
    assert normwise(y, O.spmv_crs(rp, col, val, x)) <= 1e-12
    assert k.timer("apply") == 0.0
    k.set_timers(True)
    k.run()
    assert k.timer("apply") > 0
    smax.close()
