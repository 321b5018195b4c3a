"""Pins the oracle's restatement of the reference's iterative-solver programs
(Oracle.jacobi_app / gauss_seidel_app) before it checks the GPU solvers:

1. against the printed output of the unmodified programs,
   examples/applications/{jacobi,gauss_seidel} (tests/golden/solver_apps.json,
   made by tests/golden/make_golden.py from oracle/_ref/{jacobi,gauss_seidel}):
   the BFS permutation, every residual printed with "%f", the iteration count
   and the final residual printed with 6 significant digits;
2. where the reference library was built here, against the same loops driven
   through the reference's own kernels (Reference.jacobi_app /
   gauss_seidel_app) on other sizes, right-hand sides and start vectors:
   identical iteration counts, histories and solutions.
"""
import json
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, Reference, reference_available
from smaxkernels_b200 import matrices as M

O = Oracle()
needs_ref = pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "solver_apps.json")))


def app_problem(kind):
    """The programs' problem: 10x10 Poisson (create2DPoissonMatrixCRS), b = 1;
    Jacobi permutes A by BFS first and starts from x = 1, Gauss-Seidel from 0."""
    rp, col, val = M.poisson2d_app(10)
    n = len(rp) - 1
    if kind == "jacobi":
        perm, inv, _ = O.generate_perm(rp, col, "BFS")
        rp, col, val = O.apply_mat_perm(rp, col, val, perm, inv)
        return rp, col, val, np.ones(n), np.ones(n), perm
    return rp, col, val, np.ones(n), np.zeros(n), None


@pytest.mark.parametrize("kind", ["jacobi", "gauss_seidel"])
def test_oracle_reproduces_the_programs_output(kind):
    g = GOLDEN[kind]
    rp, col, val, b, x0, perm = app_problem(kind)
    if kind == "jacobi":
        assert perm.tolist() == g["perm"]
    run = O.jacobi_app if kind == "jacobi" else O.gauss_seidel_app
    x, n_iters, norm, hist = run(rp, col, val, b, x0, g["tol"], g["max_iters"], g["check_length"])
    assert n_iters == g["converged_after"]
    assert ["%f" % h for h in hist] == g["residuals"]
    assert g["iters"] == list(range(0, n_iters + 1, g["check_length"]))
    assert "%g" % norm == g["final_residual"]


@needs_ref
@pytest.mark.parametrize("kind", ["jacobi", "gauss_seidel"])
@pytest.mark.parametrize("nx,max_iters,check_length,tol", [(10, 1000, 5, 1e-8), (24, 1000, 5, 1e-8),
                                                          (17, 37, 5, 1e-8), (12, 60, 1, 0.0),
                                                          (9, 300, 7, 1e-6)])
def test_oracle_matches_the_reference_loop(kind, nx, max_iters, check_length, tol):
    rp, col, val = M.poisson2d_app(nx)
    n = len(rp) - 1
    if kind == "jacobi":
        perm, inv, _ = O.generate_perm(rp, col, "BFS")
        rp, col, val = O.apply_mat_perm(rp, col, val, perm, inv)
    b = M.uniform_vector(n, 4)
    x0 = M.uniform_vector(n, 5)
    R = Reference()
    if kind == "jacobi":
        xo, io, no, ho = O.jacobi_app(rp, col, val, b, x0, tol, max_iters, check_length)
        xr, ir, nr, hr, _ = R.jacobi_app(rp, col, val, b, x0, tol, max_iters, check_length)
    else:
        xo, io, no, ho = O.gauss_seidel_app(rp, col, val, b, x0, tol, max_iters, check_length)
        xr, ir, nr, hr, _ = R.gauss_seidel_app(rp, col, val, b, x0, tol, max_iters, check_length)
    assert io == ir and no == nr
    np.testing.assert_array_equal(ho, hr)
    np.testing.assert_array_equal(xo, xr)


def test_infty_norm_skips_nan():
    assert O.infty_norm(np.array([np.nan, -2.0, 1.0])) == 2.0
    assert O.infty_norm(np.array([np.nan, np.nan])) == 0.0
    assert O.infty_norm(np.zeros(0)) == 0.0


def test_jacobi_peel_moves_the_last_diagonal_to_the_row_end():
    rp = np.array([0, 3, 5], np.int32)
    col = np.array([0, 1, 0, 1, 0], np.int32)
    val = np.array([5.0, 2.0, 7.0, 3.0, 1.0])
    c, v, D = O.jacobi_peel(rp, col, val)
    # row 0 holds two diagonal entries: the last one (7.0) is taken and moved
    assert c.tolist() == [0, 1, 0, 0, 1] and v.tolist() == [5.0, 2.0, 7.0, 1.0, 3.0]
    assert D.tolist() == [7.0, 3.0]
    with pytest.raises(ValueError):
        O.jacobi_peel(np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32), np.array([1.0, 1.0]))


def test_split_d_l_u_keeps_row_order():
    rp, col, val = M.poisson2d_app(4)
    (lrp, lcol, lval), (urp, ucol, uval) = O.split_d_l_u(rp, col, val)
    assert lrp[-1] + urp[-1] == len(col)
    for r in range(len(rp) - 1):
        row = col[rp[r]:rp[r + 1]]
        assert lcol[lrp[r]:lrp[r + 1]].tolist() == [c for c in row if c <= r]
        assert ucol[urp[r]:urp[r + 1]].tolist() == [c for c in row if c > r]
