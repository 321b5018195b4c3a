"""Parity of SELL-C-sigma and BCRS SpMV, their GPU conversions, and SpMM with
the oracle and the reference's golden vectors (through the C ABI)."""
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


def gpu_scs_spmv(s, x):
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


def gpu_bcrs_spmv(b, x, col_major):
    from smaxkernels_b200 import IntType, KernelType, PlatformType
    vt = b["val"].dtype
    y = np.zeros(b["n_rows"] * b["height_pad"], dtype=vt)
    smax = _iface()
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, _ft(vt))
    k = smax.kernel("k")
    k.set_mat_bcrs(True)
    k.register_A(b["n_rows"], b["n_cols"], b["n_blocks"], b["b_height"], b["b_width"], b["height_pad"],
                 b["width_pad"], b["col"], b["row_ptr"], b["val"])
    k.register_B(b["n_cols"] * b["width_pad"], np.ascontiguousarray(x, vt))
    k.register_C(b["n_rows"] * b["height_pad"], y)
    k.set_block_column_major(col_major)
    k.run()
    smax.close()
    return y


def gpu_spmm(rp, col, val, X, k_, row_major, n_cols=None, variant=0):
    from smaxkernels_b200 import IntType, KernelType, PlatformType
    n = len(rp) - 1
    Y = np.zeros(n * k_, dtype=val.dtype)
    smax = _iface()
    smax.register_kernel("k", KernelType.SPMM, PlatformType.CUDA, IntType.INT32, _ft(val.dtype))
    k = smax.kernel("k")
    if variant:
        k.set_spmv_variant(variant)
    k.register_A(n, n_cols or n, len(col), col, rp, val)
    k.register_B(n_cols or n, k_, np.ascontiguousarray(X, val.dtype))
    k.register_C(n, k_, Y)
    k.set_vec_row_major(row_major)
    k.run()
    smax.close()
    return Y


# ------------------------------------------------------------ SELL-C-sigma --
@pytest.mark.parametrize("name", G.SCS_TESTS)
def test_scs_conversion_golden_on_gpu(name):
    c = G.scs_case(name)
    smax = _iface()
    rp, col, val = c["row_ptr"], c["col"], c["val"]
    got = smax.utils.convert_crs_to_scs(len(rp) - 1, len(rp) - 1, len(col), col, rp, val, c["C"], c["sigma"])
    smax.close()
    e = c["expected"]
    for kk in ("n_rows", "n_rows_padded", "n_chunks", "n_elements", "nnz"):
        assert got[kk] == e[kk], kk
    for kk in ("chunk_ptr", "chunk_lengths", "col", "perm"):
        np.testing.assert_array_equal(got[kk], e[kk], err_msg=kk)
    np.testing.assert_array_equal(got["val"], e["val"])


@pytest.mark.parametrize("name", G.SCS_TESTS)
def test_scs_spmv_golden_matrix(name):
    c = G.scs_case(name)
    e = dict(c["expected"])
    x = np.linspace(-1.0, 1.0, e["n_cols"])
    y = gpu_scs_spmv(e, x)
    y_crs = O.spmv_crs(c["row_ptr"], c["col"], c["val"], x)
    assert G.almost_equal(y[e["perm"]], y_crs, np.float64)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("C_,sigma", [(1, 1), (2, 4), (4, 16), (8, 8), (32, 16), (32, 64), (32, 1024), (7, 3),
                                      (64, 128)])
def test_scs_random_vs_oracle(vt, C_, sigma):
    rp, col, val = rand_crs(3001, 40, 31, vt=vt, empty_frac=0.1, long_rows=(900,))
    n = len(rp) - 1
    smax = _iface()
    got = smax.utils.convert_crs_to_scs(n, n, len(col), col, rp, val, C_, sigma)
    smax.close()
    ref = O.scs(rp, col, val, C_, sigma)
    for kk in ("n_rows_padded", "n_chunks", "n_elements"):
        assert got[kk] == ref[kk]
    for kk in ("chunk_ptr", "chunk_lengths", "perm", "col", "val"):
        # the oracle and the GPU both break length ties by ascending row
        np.testing.assert_array_equal(got[kk], ref[kk], err_msg=kk)
    x = np.random.default_rng(32).uniform(-1, 1, n).astype(vt)
    y = gpu_scs_spmv(got, x)
    y_ref = O.spmv_crs(rp, col, val, x)
    assert normwise(y[got["perm"]], y_ref) <= tol(vt)


@pytest.mark.parametrize("C_,sigma", [(32, 1024), (32, 4096), (32, 8192), (8, 64), (4, 17), (2, 16), (1, 1),
                                      (32, 1 << 20)])
def test_scs_conversion_window_order_matches_oracle(C_, sigma):
    """Every array bit-exact with the oracle, whose window order is the
    reference's std::sort order (pinned in tests/test_scs_sort_order.py):
    shared-memory windows (<= 4096 rows) and in-place global-memory windows."""
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.lognormal_random(1 << 16, seed=11)
    n = len(rp) - 1
    smax = _iface()
    got = smax.utils.convert_crs_to_scs(n, n, len(col), col, rp, val, C_, sigma)
    smax.close()
    ref = O.scs(rp, col, val, C_, sigma)
    for kk in ("chunk_ptr", "chunk_lengths", "perm", "col", "val"):
        np.testing.assert_array_equal(got[kk], ref[kk], err_msg=kk)


@pytest.mark.parametrize("n", [256, 2048, 6000])
def test_scs_conversion_heapsort_fallback_matches_oracle(n):
    """Windows crafted to reach introsort's heapsort fallback, with equal
    lengths (tests/sort_adversary.py); 6000 rows take the global-memory path."""
    from sort_adversary import heap_row_lengths
    lens = np.asarray(heap_row_lengths(n), np.int64)
    rng = np.random.default_rng(12)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    col = np.concatenate([np.sort(rng.choice(n, int(l), replace=False)) for l in lens]).astype(np.int32)
    val = rng.uniform(-1, 1, len(col))
    for C_, sigma in ((1, n), (4, n)):
        smax = _iface()
        got = smax.utils.convert_crs_to_scs(n, n, len(col), col, rp, val, C_, sigma)
        smax.close()
        ref = O.scs(rp, col, val, C_, sigma)
        for kk in ("chunk_ptr", "chunk_lengths", "perm", "col", "val"):
            np.testing.assert_array_equal(got[kk], ref[kk], err_msg=f"{kk} C={C_} sigma={sigma}")


@pytest.mark.slow
@pytest.mark.parametrize("vt", [np.float64, np.float32])
def test_scs_config1_full_size(vt):
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.lognormal_random(1 << 22, dtype=vt)
    n = len(rp) - 1
    smax = _iface()
    got = smax.utils.convert_crs_to_scs(n, n, len(col), col, rp, val, 32, 1024)
    smax.close()
    ref = O.scs(rp, col, val, 32, 1024)
    for kk in ("chunk_ptr", "chunk_lengths", "perm", "col", "val"):
        np.testing.assert_array_equal(got[kk], ref[kk], err_msg=kk)
    assert got["n_elements"] == ref["n_elements"]
    x = M.uniform_vector(n, 1, dtype=vt)
    y = gpu_scs_spmv(got, x)
    y_ref = O.spmv_crs(rp, col, val.astype(np.float64), x.astype(np.float64))
    assert normwise(y[got["perm"]], y_ref) <= tol(vt)


# -------------------------------------------------------------------- BCRS --
@pytest.mark.parametrize("name", G.BCRS_CONV_TESTS)
def test_bcrs_conversion_golden_on_gpu(name):
    c = G.bcrs_conv_case(name)
    smax = _iface()
    rp = c["row_ptr"]
    b = smax.utils.convert_crs_to_bcrs(len(rp) - 1, c["n_cols"], len(c["col"]), c["col"], rp, c["val"], c["bh"],
                                       c["bw"], c["hpad"], c["wpad"], c["col_major"])
    smax.close()
    e = c["expected"]
    assert (b["n_rows"], b["n_cols"], b["n_blocks"]) == (e["n_rows"], e["n_cols"], e["n_blocks"])
    np.testing.assert_array_equal(b["row_ptr"], e["row_ptr"])
    np.testing.assert_array_equal(b["col"], e["col"])
    np.testing.assert_array_equal(b["val"], e["val"])


def test_bcrs_spmv_golden():
    c = G.bcrs_spmv_case()
    b = {k: c[k] for k in ("n_rows", "n_cols", "n_blocks", "b_height", "b_width", "height_pad", "width_pad",
                           "row_ptr", "col", "val")}
    y = gpu_bcrs_spmv(b, c["x"], c["col_major"])
    assert G.almost_equal(y, c["y"], np.float64)


@pytest.mark.parametrize("order", ["col_major", "row_major"])
def test_bcrs_laplace_golden_on_gpu(order):
    f = G.laplace()
    rp, col, val, x = (np.array(f[k]) for k in ("row_ptr", "col", "val", "x"))
    rp, col = rp.astype(np.int32), col.astype(np.int32)
    smax = _iface()
    b = smax.utils.convert_crs_to_bcrs(f["n"], f["n"], len(col), col, rp, val, f["bh"], f["bw"], f["hpad"],
                                       f["wpad"], order == "col_major")
    smax.close()
    e = f["bcrs"][order]
    np.testing.assert_array_equal(b["row_ptr"], e["row_ptr"])
    np.testing.assert_array_equal(b["col"], e["col"])
    np.testing.assert_array_equal(b["val"], np.array(e["val"]))
    y = gpu_bcrs_spmv(b, x, order == "col_major")
    assert G.almost_equal(y, e["y"], np.float64)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("shape", [(4, 4, 4, 4), (2, 8, 2, 8), (1, 1, 1, 1), (3, 5, 4, 6), (4, 4, 8, 8),
                                   (2, 2, 2, 2), (8, 4, 8, 4)])
@pytest.mark.parametrize("col_major", [False, True])
def test_bcrs_random_vs_oracle(vt, shape, col_major):
    bh, bw, hp, wp = shape
    n = 120 * bh
    nc = 90 * bw
    rp, col, val = rand_crs(n, 30, 41, vt=vt, n_cols=nc, empty_frac=0.1)
    smax = _iface()
    b = smax.utils.convert_crs_to_bcrs(n, nc, len(col), col, rp, val, bh, bw, hp, wp, col_major)
    smax.close()
    ref = O.bcrs(rp, col, val, nc, bh, bw, hp, wp, col_major)
    for kk in ("row_ptr", "col", "val"):
        np.testing.assert_array_equal(b[kk], ref[kk], err_msg=kk)
    x = np.random.default_rng(42).uniform(-1, 1, (nc // bw) * wp).astype(vt)
    y = gpu_bcrs_spmv(b, x, col_major)
    y_ref = O.spmv_bcrs(ref["n_rows"], bh, bw, hp, wp, ref["row_ptr"], ref["col"], ref["val"], col_major, x)
    rows = np.concatenate([np.arange(r * hp, r * hp + bh) for r in range(ref["n_rows"])])
    assert normwise(y[rows], y_ref[rows]) <= tol(vt)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("shape", [(4, 4, 4, 4), (2, 2, 2, 2), (8, 8, 8, 8), (3, 3, 4, 4)])
@pytest.mark.parametrize("col_major", [False, True])
def test_bcrs_long_block_rows_vs_oracle(vt, shape, col_major):
    """Block rows of many blocks (the bulk-copy stream path): warp tasks of
    several block rows, chunks that end inside a row, empty block rows and
    one block row longer than a task."""
    bh, bw, hp, wp = shape
    n = 600 * bh
    nc = 700 * bw
    rp, col, val = rand_crs(n, 120, 43, vt=vt, n_cols=nc, empty_frac=0.15, long_rows=(2500,))
    smax = _iface()
    b = smax.utils.convert_crs_to_bcrs(n, nc, len(col), col, rp, val, bh, bw, hp, wp, col_major)
    smax.close()
    x = np.random.default_rng(44).uniform(-1, 1, (nc // bw) * wp).astype(vt)
    y = gpu_bcrs_spmv(b, x, col_major)
    y_ref = O.spmv_bcrs(b["n_rows"], bh, bw, hp, wp, b["row_ptr"], b["col"], b["val"], col_major, x)
    rows = np.concatenate([np.arange(r * hp, r * hp + bh) for r in range(b["n_rows"])])
    assert normwise(y[rows], y_ref[rows]) <= tol(vt)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("col_major", [False, True])
@pytest.mark.parametrize("side", [32, 96])
def test_bcrs_short_block_rows_laplace(vt, col_major, side):
    """The 7-point Laplacian in 4x4 blocks: under two warp steps per block row,
    so a lane group per block row (odd and even block counts per row).  At
    32^3 the block values fit in half of L2 and load with the default cache
    policy; at 96^3 (99-198 MB of values) they stream evict-first."""
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace3d_7pt(side, dtype=vt)
    n = len(rp) - 1
    smax = _iface()
    b = smax.utils.convert_crs_to_bcrs(n, n, len(col), col, rp, val, 4, 4, 4, 4, col_major)
    smax.close()
    x = np.random.default_rng(45).uniform(-1, 1, n).astype(vt)
    y = gpu_bcrs_spmv(b, x, col_major)
    y_ref = O.spmv_bcrs(b["n_rows"], 4, 4, 4, 4, b["row_ptr"], b["col"], b["val"], col_major, x)
    assert normwise(y, y_ref) <= tol(vt)
    assert normwise(y, O.spmv_crs(rp, col, val.astype(np.float64), x.astype(np.float64))) <= tol(vt)


def test_bcrs_conversion_rejects_bad_blocks():
    from smaxkernels_b200 import SmaxError
    rp, col, val = rand_crs(10, 3, 1)
    smax = _iface()
    with pytest.raises(SmaxError, match="divide"):
        smax.utils.convert_crs_to_bcrs(10, 10, len(col), col, rp, val, 4, 4, 4, 4, False)
    with pytest.raises(SmaxError, match="padding"):
        smax.utils.convert_crs_to_bcrs(10, 10, len(col), col, rp, val, 2, 2, 2, 1, False)
    smax.close()


# -------------------------------------------------------------------- SpMM --
@pytest.mark.parametrize("name", ["spmm_test", "spmm_rowmaj_test"])
def test_spmm_golden(name):
    c = G.spmm_case(name)
    Y = gpu_spmm(c["row_ptr"], c["col"], c["val"], c["X"], c["k"], c["row_major"])
    assert G.almost_equal(Y, c["Y"], np.float64)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("k_", [1, 2, 3, 4, 8, 16, 17, 32, 64, 100, 128, 256])
@pytest.mark.parametrize("row_major", [True, False])
def test_spmm_random_vs_oracle(vt, k_, row_major):
    rp, col, val = rand_crs(1500, 25, 51, vt=vt, empty_frac=0.1, long_rows=(1400,))
    X = np.random.default_rng(52).uniform(-1, 1, 1500 * k_).astype(vt)
    Y = gpu_spmm(rp, col, val, X, k_, row_major)
    Y_ref = O.spmm(rp, col, val, X, k_, row_major=row_major)
    assert normwise(Y, Y_ref) <= tol(vt)
    Y64 = O.spmm(rp, col, val.astype(np.float64), X.astype(np.float64), k_, row_major=row_major)
    assert normwise(Y, Y64) <= tol(vt)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("k_", [1, 3, 16, 64, 100])
def test_spmm_row_major_kernels_agree(vt, k_):
    """The all-rows grid and the per-SM row walks compute each row with the
    same group and the same order of products: bit-identical results."""
    rp, col, val = rand_crs(20000, 9, 61, vt=vt, empty_frac=0.05, long_rows=(3000,))
    X = np.random.default_rng(62).uniform(-1, 1, 20000 * k_).astype(vt)
    Y1 = gpu_spmm(rp, col.copy(), val.copy(), X, k_, True, variant=1)
    Y2 = gpu_spmm(rp, col.copy(), val.copy(), X, k_, True, variant=2)
    np.testing.assert_array_equal(Y1, Y2)
    assert normwise(Y2, O.spmm(rp, col, val, X, k_, row_major=True)) <= tol(vt)


@pytest.mark.slow
@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("k_", [16, 64])
def test_spmm_config2_stencil27(vt, k_):
    from smaxkernels_b200 import matrices as M
    nx = 128 if k_ == 16 else 64  # the oracle needs seconds per k; 64^3 keeps k=64 short
    rp, col, val = M.stencil27(nx, dtype=vt)
    n = len(rp) - 1
    X = np.random.default_rng(2).uniform(-1, 1, n * k_).astype(vt)
    Y = gpu_spmm(rp, col, val, X, k_, True)
    Y_ref = O.spmm(rp, col, val.astype(np.float64), X.astype(np.float64), k_, row_major=True)
    assert normwise(Y, Y_ref) <= tol(vt)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("x0", [1.5, np.inf, np.nan])
def test_scs_padding_skip_matches_reference_semantics(vt, x0):
    """The SELL task kernel skips each row's padding (column 0, value 0 past its
    last other stored entry) when x[0] is finite.  With x[0] infinite or NaN it
    uses every stored entry, as the reference's SELL loop does, so 0 * x[0]
    makes NaN in every row that holds padding -- the oracle's SELL product
    (over all stored entries) is the reference here.  Some rows end with an
    explicit zero in column 0, which the kernel may skip with a finite x[0]."""
    rng = np.random.default_rng(46)
    n = 3000
    lens = rng.integers(1, 40, n)
    lens[::50] = 300
    rows = []
    for r, l in enumerate(lens):
        c = np.sort(rng.choice(np.arange(1, n), int(l), replace=False)).astype(np.int32)
        if r % 7 == 0:
            c = np.concatenate([c[:-1], [0]]).astype(np.int32)  # ends in column 0
        rows.append(c)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    col = np.concatenate(rows).astype(np.int32)
    val = rng.uniform(-1, 1, len(col)).astype(vt)
    val[rp[1:][::7] - 1] = 0.0  # those column-0 entries are explicit zeros
    smax = _iface()
    s = smax.utils.convert_crs_to_scs(n, n, len(col), col, rp, val, 32, 128)
    smax.close()
    x = rng.uniform(-1, 1, n).astype(vt)
    x[0] = x0
    y = gpu_scs_spmv(s, x)
    xx = np.zeros(max(s["n_rows_padded"], n), vt)
    xx[:n] = x
    y_ref = O.spmv_scs(32, s["chunk_ptr"], s["chunk_lengths"], s["col"], s["val"], xx, s["n_rows_padded"])
    y, y_ref = y[: s["n_rows_padded"]], y_ref[: s["n_rows_padded"]]
    np.testing.assert_array_equal(np.isnan(y), np.isnan(y_ref))
    if np.isfinite(x0):
        assert not np.isnan(y).any()
    else:
        assert np.isnan(y).any()
    fin = ~np.isnan(y_ref)
    assert normwise(y[fin], y_ref[fin]) <= tol(vt)


def test_scs_split_chunks_repeated_products():
    """Chunks longer than 32 columns are split over several warps and the
    chunk's last warp adds their partial sums; its counter must be back at 0
    for the next product.  Five products on one kernel object, x changing."""
    from smaxkernels_b200 import IntType, KernelType, PlatformType
    rp, col, val = rand_crs(4000, 30, 47, empty_frac=0.05, long_rows=(1500, 700, 300))
    n = len(rp) - 1
    smax = _iface()
    s = smax.utils.convert_crs_to_scs(n, n, len(col), col, rp, val, 32, 256)
    assert max(s["chunk_lengths"]) > 32
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, _ft(val.dtype))
    k = smax.kernel("k")
    k.set_mat_scs(True)
    vs = max(s["n_rows_padded"], n)
    xx = np.zeros(vs)
    y = np.zeros(vs)
    k.register_A(s["C"], s["sigma"], s["n_rows"], s["n_rows_padded"], n, s["n_chunks"], s["n_elements"],
                 s["nnz"], s["chunk_ptr"], s["chunk_lengths"], s["col"], s["val"], s["perm"])
    k.register_B(vs, xx)
    k.register_C(vs, y)
    rng = np.random.default_rng(48)
    for _ in range(5):
        xx[:n] = rng.uniform(-1, 1, n)
        k.run()
        assert normwise(y[s["perm"]], O.spmv_crs(rp, col, val, xx[:n])) <= 1e-12
    smax.close()
