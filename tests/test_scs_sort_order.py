"""The SELL-C-sigma window order of the oracle is the reference's std::sort
order, pinned against the unmodified reference (oracle/_ref/libsmax_ref.so):
lognormal row lengths (many equal lengths per window) at every sigma regime
-- insertion sort only (sigma <= 16), introsort with the final insertion
pass, windows longer than the whole matrix -- and crafted windows that reach
introsort's heapsort fallback with equal lengths (tests/sort_adversary.py).
A stable order differs from the reference on these inputs, so the checks
have teeth.  The GPU conversion is checked against the same cases in
tests/test_gpu_formats.py.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, Reference, reference_available
from sort_adversary import heap_row_lengths, uses_heap

needs_ref = pytest.mark.skipif(not reference_available(), reason="oracle/_ref/libsmax_ref.so is not built")
O = Oracle()


def lognormal_case(n, seed=11):
    from smaxkernels_b200 import matrices as M
    return M.lognormal_random(n, seed=seed)


def rows_with_lengths(lens, n_cols, seed=12):
    rng = np.random.default_rng(seed)
    lens = np.asarray(lens, np.int64)
    rp = np.zeros(len(lens) + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    col = np.concatenate([np.sort(rng.choice(n_cols, int(l), replace=False)) for l in lens]).astype(np.int32)
    return rp, col, rng.uniform(-1, 1, len(col))


def stable_perm(rp, sigma):
    """perm[old] = new under a STABLE descending sort of every window."""
    lens = np.diff(rp)
    n = len(lens)
    perm = np.empty(n, np.int64)
    for w in range(0, n, sigma):
        order = w + np.argsort(-lens[w:w + sigma], kind="stable")
        perm[order] = np.arange(w, w + len(order))
    return perm


@needs_ref
@pytest.mark.parametrize("C_,sigma", [(32, 1024), (32, 4096), (8, 64), (4, 17), (2, 16), (1, 1), (32, 1 << 20)])
def test_oracle_window_order_is_the_references(C_, sigma):
    R = Reference()
    rp, col, val = lognormal_case(1 << 16)
    a, b = O.scs(rp, col, val, C_, sigma), R.scs(rp, col, val, C_, sigma)
    for k in ("chunk_ptr", "chunk_lengths", "perm", "col", "val"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    if sigma > 16:  # where the order of ties is the library's, a stable sort disagrees
        assert np.count_nonzero(stable_perm(rp, sigma)[: len(rp) - 1] != b["perm"]) > 0


@needs_ref
@pytest.mark.parametrize("n", [256, 1024, 2048])
def test_oracle_heapsort_fallback_with_ties(n):
    lens = heap_row_lengths(n)
    assert uses_heap([-l for l in lens]), "the crafted window must reach the heapsort fallback"
    assert len(set(lens)) < n, "and hold equal lengths"
    R = Reference()
    rp, col, val = rows_with_lengths(lens, n)
    for C_, sigma in ((1, n), (4, n), (1, n // 2)):
        a, b = O.scs(rp, col, val, C_, sigma), R.scs(rp, col, val, C_, sigma)
        for k in ("chunk_ptr", "chunk_lengths", "perm", "col", "val"):
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"{k} C={C_} sigma={sigma}")
    assert np.count_nonzero(stable_perm(rp, n) != R.scs(rp, col, val, 1, n)["perm"]) > 0
