"""Parity of the GPU Gustavson SpGEMM with the oracle and the reference's golden
vectors: C's pattern (row_ptr and the FIRST-TOUCH column order in each row) is
bit-exact, values within the normwise tolerance."""
import numpy as np
import pytest

import golden_cases as G
from helpers import normwise, rand_crs, tol
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
O = Oracle()


def gpu_spgemm(A, B, a_n_cols, b_n_cols):
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    (arp, acol, aval), (brp, bcol, bval) = A, B
    ft = FloatType.FLOAT32 if aval.dtype == np.float32 else FloatType.FLOAT64
    smax = Interface()
    smax.register_kernel("g", KernelType.SPGEMM, PlatformType.CUDA, IntType.INT32, ft)
    k = smax.kernel("g")
    k.register_A(len(arp) - 1, a_n_cols, len(acol), acol.astype(np.int32), arp.astype(np.int32), aval)
    k.register_B(len(brp) - 1, b_n_cols, len(bcol), bcol.astype(np.int32), brp.astype(np.int32), bval)
    k.register_C()
    k.run()
    res = k.result()
    smax.close()
    return res


@pytest.mark.parametrize("name", ["spgemmAA_test", "spgemmAB_test"])
def test_spgemm_golden(name):
    """spgemmAA_test uses uint16 indices in the reference; this platform runs
    int32 indices, the pattern and values are the same."""
    c = G.spgemm_case(name)
    n_rows, n_cols, nnz, rp, col, val = gpu_spgemm(c["A"], c["B"], c["b_n_cols"], c["b_n_cols"])
    assert (n_rows, n_cols, nnz) == (len(c["C"][0]) - 1, c["b_n_cols"], len(c["C"][1]))
    np.testing.assert_array_equal(rp, c["C"][0])
    np.testing.assert_array_equal(col, c["C"][1])
    assert G.almost_equal(val, c["C"][2], np.float32)


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("shape", ["square", "rect", "empty_rows"])
def test_spgemm_random_vs_oracle(vt, shape):
    if shape == "square":
        A = rand_crs(2000, 12, 101, vt=vt)
        B = rand_crs(2000, 12, 102, vt=vt)
        a_nc, b_nc = 2000, 2000
    elif shape == "rect":
        A = rand_crs(1500, 10, 103, vt=vt, n_cols=800)
        B = rand_crs(800, 15, 104, vt=vt, n_cols=3000)
        a_nc, b_nc = 800, 3000
    else:
        A = rand_crs(2000, 8, 105, vt=vt, empty_frac=0.5)
        B = rand_crs(2000, 8, 106, vt=vt, empty_frac=0.5)
        a_nc, b_nc = 2000, 2000
    n_rows, n_cols, nnz, rp, col, val = gpu_spgemm(A, B, a_nc, b_nc)
    orp, ocol, oval = O.spgemm(*A, *B, b_nc)
    assert (n_rows, n_cols) == (len(A[0]) - 1, b_nc)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(col, ocol)
    assert normwise(val, oval) <= tol(vt)


@pytest.mark.parametrize("maxlen", [40, 90, 300])
def test_spgemm_heavy_rows(maxlen):
    """Rows with hundreds to tens of thousands of products: the CTA and the
    global-workspace paths."""
    A = rand_crs(600, maxlen, 111, long_rows=(590, 599))
    B = rand_crs(600, maxlen, 112, long_rows=(580,))
    n_rows, n_cols, nnz, rp, col, val = gpu_spgemm(A, B, 600, 600)
    orp, ocol, oval = O.spgemm(*A, *B, 600)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(col, ocol)
    assert normwise(val, oval) <= 1e-12


@pytest.mark.slow
def test_spgemm_config2_laplace96():
    from smaxkernels_b200 import matrices as M
    A = M.laplace3d_7pt(96)
    n_rows, n_cols, nnz, rp, col, val = gpu_spgemm(A, A, 96 ** 3, 96 ** 3)
    orp, ocol, oval = O.spgemm(*A, *A, 96 ** 3)
    assert nnz == 21_732_480
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(col, ocol)
    assert normwise(val, oval) <= 1e-12


def _shuffle_rows(rp, col, val, seed):
    """The same matrix with each row's entries in a random order."""
    rng = np.random.default_rng(seed)
    col, val = col.copy(), val.copy()
    for r in range(len(rp) - 1):
        a, b = rp[r], rp[r + 1]
        o = rng.permutation(b - a)
        col[a:b], val[a:b] = col[a:b][o], val[a:b][o]
    return rp, col, val


@pytest.mark.parametrize("sorted_b", [True, False])
def test_spgemm_merge_and_hash_paths_vs_oracle(sorted_b):
    """Rows of A with at most 8 entries and 64 products take the merge path
    when every row of B has increasing columns; with B's rows shuffled every
    row takes the hash paths.  Both give the first-touch pattern and the
    product-order sums of the oracle.  The matrix mixes rows at the merge
    limits (8 entries, products up to 64), rows of 9+ entries, empty rows of
    A and of B."""
    rng = np.random.default_rng(120)
    n = 3000
    lens = rng.integers(0, 10, n)
    lens[::7] = 8
    lens[::11] = 0
    rows = [np.sort(rng.choice(n, int(l), replace=False)) for l in lens]
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    col = np.concatenate(rows).astype(np.int32)
    A = (rp, col, rng.uniform(-1, 1, len(col)))
    blens = rng.integers(0, 9, n)
    blens[::13] = 0
    brows = [np.sort(rng.choice(n, int(l), replace=False)) for l in blens]
    brp = np.zeros(n + 1, np.int32)
    brp[1:] = np.cumsum(blens)
    B = (brp, np.concatenate(brows).astype(np.int32), rng.uniform(-1, 1, int(blens.sum())))
    if not sorted_b:
        B = _shuffle_rows(*B, seed=121)
    n_rows, n_cols, nnz, crp, ccol, cval = gpu_spgemm(A, B, n, n)
    orp, ocol, oval = O.spgemm(*A, *B, n)
    np.testing.assert_array_equal(crp, orp)
    np.testing.assert_array_equal(ccol, ocol)
    assert normwise(cval, oval) <= 1e-12


def test_spgemm_merge_path_rectangular():
    A = rand_crs(1200, 8, 122, n_cols=700)
    B = rand_crs(700, 8, 123, n_cols=2500)
    n_rows, n_cols, nnz, rp, col, val = gpu_spgemm(A, B, 700, 2500)
    orp, ocol, oval = O.spgemm(*A, *B, 2500)
    assert (n_rows, n_cols) == (1200, 2500)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(col, ocol)
    assert normwise(val, oval) <= 1e-12


@pytest.mark.parametrize("case", ["disjoint64", "overlapping"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_spgemm_direct_merge_path(case, dtype):
    """Every row of A on the merge path, so C is written straight from the
    second merge pass, one warp staging its 32 rows in shared memory.
    "disjoint64": every non-empty row of A selects 8 B rows with disjoint
    columns, 64 distinct entries per row of C -- the largest staging size.
    "overlapping": random rows of at most 8 entries over short sorted B rows.
    Both have empty rows and a row count that ends in a partial warp."""
    rng = np.random.default_rng(124 if case == "disjoint64" else 125)
    n = 32 * 37 + 19
    if case == "disjoint64":
        nb = 700
        brp = np.arange(nb + 1, dtype=np.int32) * 8
        bcol = (np.arange(nb)[:, None] * 8 + np.arange(8)[None, :]).reshape(-1).astype(np.int32)
        b_n_cols = 8 * nb
        lens = np.full(n, 8)
        lens[::9] = 0
        rows = [rng.choice(nb, 8, replace=False) if l else np.zeros(0, int) for l in lens]
    else:
        nb = 900
        blens = rng.integers(0, 9, nb)
        blens[::17] = 0
        brp = np.zeros(nb + 1, np.int32)
        brp[1:] = np.cumsum(blens)
        bcol = np.concatenate([np.sort(rng.choice(nb, int(l), replace=False)) for l in blens]).astype(np.int32)
        b_n_cols = nb
        lens = rng.integers(0, 9, n)
        lens[::5] = 0
        rows = [rng.choice(nb, int(l), replace=False) for l in lens]
    bval = rng.uniform(-1, 1, len(bcol)).astype(dtype)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(r) for r in rows])
    col = np.concatenate(rows).astype(np.int32)
    A = (rp, col, rng.uniform(-1, 1, len(col)).astype(dtype))
    B = (brp, bcol, bval)
    n_rows, n_cols, nnz, crp, ccol, cval = gpu_spgemm(A, B, nb, b_n_cols)
    orp, ocol, oval = O.spgemm(*A, *B, b_n_cols)
    if case == "disjoint64":
        assert np.diff(orp).max() == 64
    np.testing.assert_array_equal(crp, orp)
    np.testing.assert_array_equal(ccol, ocol)
    assert normwise(cval, oval) <= tol(dtype)


def test_spgemm_direct_hint_falls_back_to_classified_rows():
    """After an apply on the direct merge path, the kernel object's next apply
    tries that path first, and its pass 1 checks every row.  Four runs on one
    kernel object, with operands of unchanged sizes:
    - B sorted: the direct path;
    - B's rows shuffled: no row may merge, so the rows are classified again;
    - B sorted again: the direct path once more;
    - one row of A given 9 entries: classified again.
    Every run matches the oracle."""
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    rng = np.random.default_rng(126)
    n = 2000
    lens = rng.integers(0, 9, n)
    rows = [rng.choice(n, int(l), replace=False) for l in lens]
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    A = (rp, np.concatenate(rows).astype(np.int32), rng.uniform(-1, 1, int(lens.sum())))
    blens = rng.integers(0, 9, n)
    brp = np.zeros(n + 1, np.int32)
    brp[1:] = np.cumsum(blens)
    bcol = np.concatenate([np.sort(rng.choice(n, int(l), replace=False)) for l in blens]).astype(np.int32)
    B = (brp, bcol, rng.uniform(-1, 1, len(bcol)))
    A9 = (np.concatenate([[0], np.cumsum(np.where(np.arange(n) == 5, 9, lens))]).astype(np.int32),
          np.concatenate([rng.choice(n, 9, replace=False) if r == 5 else rows[r] for r in range(n)]).astype(np.int32),
          None)
    A9 = (A9[0], A9[1], rng.uniform(-1, 1, len(A9[1])))
    smax = Interface()
    smax.register_kernel("g", KernelType.SPGEMM, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("g")
    for a, b in ((A, B), (A, _shuffle_rows(*B, seed=127)), (A, B), (A9, B)):
        k.register_A(n, n, len(a[1]), a[1], a[0], a[2])
        k.register_B(n, n, len(b[1]), b[1], b[0], b[2])
        k.register_C()
        k.run()
        _, _, _, crp, ccol, cval = k.result()
        orp, ocol, oval = O.spgemm(*a, *b, n)
        np.testing.assert_array_equal(crp, orp)
        np.testing.assert_array_equal(ccol, ocol)
        assert normwise(cval, oval) <= 1e-12
    smax.close()


def test_spgemm_timers_off():
    """With the timers off SpGEMM records no phase events: its phase timers
    stay 0 and C is unchanged."""
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    A = rand_crs(1500, 8, 128)
    smax = Interface()
    smax.register_kernel("g", KernelType.SPGEMM, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("g")
    k.set_timers(False)
    rp, col, val = A
    k.register_A(1500, 1500, len(col), col, rp, val)
    k.register_B(1500, 1500, len(col), col, rp, val)
    for _ in range(2):
        k.register_C()
        k.run()
        _, _, _, crp, ccol, cval = k.result()
        orp, ocol, oval = O.spgemm(*A, *A, 1500)
        np.testing.assert_array_equal(crp, orp)
        np.testing.assert_array_equal(ccol, ocol)
        assert normwise(cval, oval) <= 1e-12
    for name in ("apply", "Symbolic_Setup", "Fused_Gustavson", "Alloc_C", "Compress"):
        assert k.timer(name) == 0.0, name
    smax.close()


def test_spgemm_direct_path_with_a_growing_and_shrinking_product():
    """Three runs on one kernel object, each on the direct merge path from the
    last run's hint: rows of A with at most 4 entries, then up to 8 (a larger
    C: more entries and a fuller warp to stage), then at most 4 again.  C's
    arrays and the staging size follow each product; every run matches the
    oracle."""
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    rng = np.random.default_rng(129)
    n = 2500
    blens = rng.integers(1, 9, n)
    brp = np.zeros(n + 1, np.int32)
    brp[1:] = np.cumsum(blens)
    bcol = np.concatenate([np.sort(rng.choice(n, int(l), replace=False)) for l in blens]).astype(np.int32)
    B = (brp, bcol, rng.uniform(-1, 1, len(bcol)))

    def make_a(max_len, seed):
        r = np.random.default_rng(seed)
        lens = r.integers(0, max_len + 1, n)
        rows = [r.choice(n, int(l), replace=False) for l in lens]
        rp = np.zeros(n + 1, np.int32)
        rp[1:] = np.cumsum(lens)
        col = np.concatenate(rows).astype(np.int32)
        return rp, col, r.uniform(-1, 1, len(col))

    small, big = make_a(4, 130), make_a(8, 131)
    smax = Interface()
    smax.register_kernel("g", KernelType.SPGEMM, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("g")
    k.register_B(n, n, len(B[1]), B[1], B[0], B[2])
    nnzs = []
    for a in (small, big, small):
        k.register_A(n, n, len(a[1]), a[1], a[0], a[2])
        k.register_C()
        k.run()
        _, _, nnz, crp, ccol, cval = k.result()
        orp, ocol, oval = O.spgemm(*a, *B, n)
        np.testing.assert_array_equal(crp, orp)
        np.testing.assert_array_equal(ccol, ocol)
        assert normwise(cval, oval) <= 1e-12
        nnzs.append(nnz)
    assert nnzs[1] > nnzs[0]
    smax.close()
