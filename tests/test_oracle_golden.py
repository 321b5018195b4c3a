"""Pins the CPU oracle (oracle/smax_oracle.c) before it is trusted as a checker:

1. against every known-answer vector of the reference's hot-path unit tests
   (tests/golden/*.json, extracted from examples/tests/*.hpp), and
2. where the reference itself was built here (oracle/_ref), against the
   reference on seeded random inputs.
"""
import numpy as np
import pytest

import golden_cases as G
from oracle.oracle import Oracle, Reference, reference_available

O = Oracle()
needs_ref = pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")


def test_spmv_crs_golden():
    c = G.spmv_case()
    assert G.almost_equal(O.spmv_crs(c["row_ptr"], c["col"], c["val"], c["x"]), c["y"], c["val"].dtype)


@pytest.mark.parametrize("name", G.SCS_TESTS)
def test_scs_conversion_golden(name):
    c = G.scs_case(name)
    got = O.scs(c["row_ptr"], c["col"], c["val"], c["C"], c["sigma"])
    e = c["expected"]
    for k in ("n_rows", "n_rows_padded", "n_chunks", "n_elements", "nnz"):
        assert got[k] == e[k], k
    for k in ("chunk_ptr", "chunk_lengths", "col", "perm"):
        np.testing.assert_array_equal(got[k], e[k], err_msg=k)
    assert G.almost_equal(got["val"], e["val"], e["val"].dtype)


@pytest.mark.parametrize("name", G.SCS_TESTS)
def test_scs_spmv_golden_unpermuted(name):
    """SCS SpMV on the converted matrix equals CRS SpMV after y_scs[perm[i]]."""
    c = G.scs_case(name)
    s = O.scs(c["row_ptr"], c["col"], c["val"], c["C"], c["sigma"])
    n = s["n_rows"]
    x = np.linspace(-1.0, 1.0, n)
    y_scs = O.spmv_scs(s["C"], s["chunk_ptr"], s["chunk_lengths"], s["col"], s["val"], x, s["n_rows_padded"])
    y_crs = O.spmv_crs(c["row_ptr"], c["col"], c["val"], x)
    np.testing.assert_allclose(y_scs[s["perm"]], y_crs, rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("name", G.BCRS_CONV_TESTS)
def test_bcrs_conversion_golden(name):
    c = G.bcrs_conv_case(name)
    got = O.bcrs(c["row_ptr"], c["col"], c["val"], c["n_cols"], c["bh"], c["bw"], c["hpad"], c["wpad"],
                 c["col_major"])
    e = c["expected"]
    assert (got["n_rows"], got["n_cols"], got["n_blocks"]) == (e["n_rows"], e["n_cols"], e["n_blocks"])
    np.testing.assert_array_equal(got["row_ptr"], e["row_ptr"])
    np.testing.assert_array_equal(got["col"], e["col"])
    assert G.almost_equal(got["val"], e["val"], np.float64)


def test_bcrs_spmv_golden():
    c = G.bcrs_spmv_case()
    y = O.spmv_bcrs(c["n_rows"], c["b_height"], c["b_width"], c["height_pad"], c["width_pad"], c["row_ptr"],
                    c["col"], c["val"], c["col_major"], c["x"])
    assert G.almost_equal(y, c["y"], np.float64)


@pytest.mark.parametrize("order", ["col_major", "row_major"])
def test_bcrs_laplace_golden(order):
    f = G.laplace()
    rp, col, val, x = (np.array(f[k]) for k in ("row_ptr", "col", "val", "x"))
    b = O.bcrs(rp, col, val, f["n"], f["bh"], f["bw"], f["hpad"], f["wpad"], order == "col_major")
    e = f["bcrs"][order]
    np.testing.assert_array_equal(b["row_ptr"], e["row_ptr"])
    np.testing.assert_array_equal(b["col"], e["col"])
    assert G.almost_equal(b["val"], e["val"], np.float64)
    y = O.spmv_bcrs(b["n_rows"], f["bh"], f["bw"], f["hpad"], f["wpad"], b["row_ptr"], b["col"], b["val"],
                    order == "col_major", x)
    assert G.almost_equal(y, e["y"], np.float64)
    assert G.almost_equal(y, f["y_crs"], np.float64)


@pytest.mark.parametrize("name", ["spmm_test", "spmm_rowmaj_test"])
def test_spmm_golden(name):
    c = G.spmm_case(name)
    Y = O.spmm(c["row_ptr"], c["col"], c["val"], c["X"], c["k"], row_major=c["row_major"])
    assert G.almost_equal(Y, c["Y"], c["val"].dtype)


@pytest.mark.parametrize("name", ["spgemmAA_test", "spgemmAB_test"])
def test_spgemm_golden(name):
    c = G.spgemm_case(name)
    (arp, acol, aval), (brp, bcol, bval) = c["A"], c["B"]
    crp, ccol, cval = O.spgemm(arp, acol, aval, brp, bcol, bval, c["b_n_cols"])
    np.testing.assert_array_equal(crp, c["C"][0])
    np.testing.assert_array_equal(ccol, c["C"][1])  # first-touch order, bit-exact
    assert G.almost_equal(cval, c["C"][2], np.float32)


def test_sptrsv_golden():
    c = G.sptrsv_case()
    x = O.sptrsv(c["row_ptr"], c["col"], c["val"], c["b"])
    assert G.almost_equal(x, c["x"], np.float64)


@pytest.mark.parametrize("name", ["sptrsm_test", "sptrsm_rowmaj_test"])
def test_sptrsm_golden(name):
    c = G.sptrsm_case(name)
    X = O.sptrsm(c["row_ptr"], c["col"], c["val"], c["B"], c["k"], row_major=c["row_major"])
    assert G.almost_equal(X, c["X"], np.float64)


@pytest.mark.parametrize("name", ["perm_test_1", "perm_test_2"])
def test_perm_golden(name):
    c = G.perm_case(name)
    for typ, exp_perm, exp_val in (("BFS", c["perm_bfs"], c["val_bfs"]), ("RS", c["perm_rs"], c["val_rs"])):
        perm, inv, lvl_ptr = O.generate_perm(c["row_ptr"], c["col"], typ)
        assert len(lvl_ptr) - 1 == c["n_levels"]
        np.testing.assert_array_equal(lvl_ptr, c["lvl_ptr"])
        np.testing.assert_array_equal(perm, exp_perm)
        np.testing.assert_array_equal(perm[inv], np.arange(len(perm)))
        _, _, pval = O.apply_mat_perm(c["row_ptr"], c["col"], c["val"], perm, inv)
        np.testing.assert_array_equal(pval, exp_val)


@pytest.mark.parametrize("name", ["build_symmetric_crs_1", "build_symmetric_crs_2", "build_symmetric_crs_3"])
def test_build_symmetric_golden(name):
    c = G.symmetric_case(name)
    srp, scol = O.build_symmetric(c["row_ptr"], c["col"])
    np.testing.assert_array_equal(srp, c["sym_row_ptr"])
    np.testing.assert_array_equal(G.sort_rows(srp, scol), c["sym_col"])


# ---------------------------------------------------------------------------
# Oracle vs the reference itself on seeded random inputs
# ---------------------------------------------------------------------------
def _rand_crs(n, maxlen, seed, lower=False, vt=np.float64, n_cols=None):
    rng = np.random.default_rng(seed)
    n_cols = n_cols or n
    rows = []
    for r in range(n):
        if lower:
            k = min(int(rng.integers(0, maxlen)), r)
            c = np.sort(np.concatenate([rng.choice(r, k, replace=False) if k else np.zeros(0, int), [r]]))
        else:
            k = int(rng.integers(0, maxlen))
            c = np.sort(rng.choice(n_cols, min(k, n_cols), replace=False))
        rows.append(c)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(c) for c in rows])
    col = np.concatenate(rows).astype(np.int32) if rows else np.zeros(0, np.int32)
    val = rng.uniform(-1, 1, len(col)).astype(vt)
    if lower:
        val[rp[1:] - 1] = (4.0 + rng.uniform(0, 1, n)).astype(vt)
    return rp, col, val


@needs_ref
@pytest.mark.parametrize("vt", [np.float64, np.float32])
def test_vs_reference_spmv_spmm(vt):
    R = Reference()
    rp, col, val = _rand_crs(500, 30, 1, vt=vt)
    x = np.random.default_rng(2).uniform(-1, 1, 500).astype(vt)
    np.testing.assert_allclose(O.spmv_crs(rp, col, val, x), R.spmv_crs(rp, col, val, x), rtol=1e-5, atol=1e-5)
    X = np.random.default_rng(3).uniform(-1, 1, 500 * 7).astype(vt)
    for rm in (True, False):
        np.testing.assert_allclose(O.spmm(rp, col, val, X, 7, rm), R.spmm(rp, col, val, X, 7, rm),
                                   rtol=1e-5, atol=1e-5)


@needs_ref
def test_vs_reference_conversions():
    R = Reference()
    rp, col, val = _rand_crs(512, 40, 4)
    # every array bit-exact, including perm/col/val where the windows hold
    # more than 16 rows and std::sort's order of equal-length rows matters
    for C_, s in ((1, 1), (2, 4), (4, 16), (8, 8), (32, 16), (32, 1024), (32, 128), (4, 17), (1, 512)):
        a, b = O.scs(rp, col, val, C_, s), R.scs(rp, col, val, C_, s)
        for k in ("chunk_ptr", "chunk_lengths", "col", "val", "perm"):
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"{k} C={C_} sigma={s}")
        assert a["n_elements"] == b["n_elements"]
    for bh, bw in ((4, 4), (2, 8), (1, 1)):
        for cm in (True, False):
            a = O.bcrs(rp, col, val, 512, bh, bw, bh, bw, cm)
            b = R.bcrs(rp, col, val, 512, bh, bw, bh, bw, cm)
            for k in ("row_ptr", "col", "val"):
                np.testing.assert_array_equal(a[k], b[k])


@needs_ref
def test_vs_reference_spgemm():
    R = Reference()
    A = _rand_crs(300, 12, 5)
    B = _rand_crs(300, 12, 6)
    a = O.spgemm(*A, *B, 300)
    b = R.spgemm(*A, *B, 300, 300)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_allclose(a[2], b[2], rtol=1e-12, atol=1e-13)


@needs_ref
def test_vs_reference_levels_and_solves():
    R = Reference()
    rp, col, val = _rand_crs(400, 6, 7, lower=True)
    R.set_threads(1)
    try:
        for t in ("RS", "BFS"):
            p1, i1, l1 = O.generate_perm(rp, col, t)
            p2, i2, l2 = R.generate_perm(rp, col, t)
            np.testing.assert_array_equal(p1, p2)
            np.testing.assert_array_equal(l1, l2)
    finally:
        R.set_threads(0)
    srp1, sc1 = O.build_symmetric(rp, col)
    srp2, sc2 = R.build_symmetric(rp, col)
    np.testing.assert_array_equal(srp1, srp2)
    np.testing.assert_array_equal(sc1, sc2)
    b = np.random.default_rng(8).uniform(-1, 1, 400)
    np.testing.assert_allclose(O.sptrsv(rp, col, val, b), R.sptrsv(rp, col, val, b), rtol=1e-13, atol=1e-13)
    # level-scheduled solve on the permuted lower triangle (reference flow)
    perm, inv, lvl = O.generate_perm(rp, col, "RS")
    prp, pcol, pval = O.apply_mat_perm(rp, col, val, perm, inv)
    bp = O.apply_vec_perm(b, perm)
    np.testing.assert_allclose(O.sptrsv(prp, pcol, pval, bp, levels=lvl),
                               R.sptrsv(prp, pcol, pval, bp, levels=lvl), rtol=1e-13, atol=1e-13)
    B = np.random.default_rng(9).uniform(-1, 1, 400 * 3)
    np.testing.assert_allclose(O.sptrsm(rp, col, val, B, 3, row_major=True),
                               R.sptrsm(rp, col, val, B, 3, row_major=True), rtol=1e-13, atol=1e-13)
