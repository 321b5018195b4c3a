"""Device-resident Jacobi and Gauss-Seidel (smax_solver_*) against the oracle's
restatement of the reference's solver programs and against those programs'
printed output (tests/golden/solver_apps.json).

Tolerances: iteration counts are equal; solutions agree to 1e-12 normwise
relative (FP64), 1e-4 (FP32).  The GPU sums rows in another order, so x
differs from the oracle's in the last bits; a residual |b - A x| near the
tolerance is a difference of nearly equal numbers and carries that rounding
at ~1e-15 absolute.  Residuals are therefore compared to 1e-9 relative plus
1e-12 of the first residual, and to the programs' printed digits within their
rounding ("%f": 5e-7 absolute; "%g": 1e-5 relative).
"""
import json
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from smaxkernels_b200 import matrices as M
from smaxkernels_b200._lib import SmaxError
from smaxkernels_b200.solvers import Solver

pytestmark = pytest.mark.gpu
O = Oracle()
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "solver_apps.json")))
MODES = ["device_loop", "graph_blocks", "plain"]


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def app_problem(kind, nx=10, gpu_perm=True):
    rp, col, val = M.poisson2d_app(nx)
    n = len(rp) - 1
    if kind == "jacobi":
        if gpu_perm:
            from smaxkernels_b200 import Interface
            smax = Interface()
            perm = np.zeros(n, np.int32)
            inv = np.zeros(n, np.int32)
            smax.utils.generate_perm(n, rp, col, perm, inv, "BFS")
            prp, pcol, pval = np.zeros(n + 1, np.int32), np.zeros(len(col), np.int32), np.zeros(len(col))
            smax.utils.apply_mat_perm(n, rp, col, val, prp, pcol, pval, perm, inv)
            smax.close()
            return prp, pcol, pval, np.ones(n), np.ones(n), perm
        perm, inv, _ = O.generate_perm(rp, col, "BFS")
        prp, pcol, pval = O.apply_mat_perm(rp, col, val, perm, inv)
        return prp, pcol, pval, np.ones(n), np.ones(n), perm
    return rp, col, val, np.ones(n), np.zeros(n), None


def check_hist(h, ho):
    assert len(h) == len(ho)
    np.testing.assert_allclose(h, ho, rtol=1e-9, atol=1e-12 * max(float(ho[0]), 1e-300))


def oracle_run(kind, *a, **kw):
    return (O.jacobi_app if kind == "jacobi" else O.gauss_seidel_app)(*a, **kw)


@pytest.mark.parametrize("kind", ["jacobi", "gauss_seidel"])
@pytest.mark.parametrize("mode", MODES)
def test_the_programs_problem(kind, mode):
    g = GOLDEN[kind]
    rp, col, val, b, x0, perm = app_problem(kind)
    if perm is not None:
        assert perm.tolist() == g["perm"]
    x = x0.copy()
    with Solver(kind, rp, col, val) as s:
        st = s.solve(b, x, tol=g["tol"], max_iters=g["max_iters"], check_length=g["check_length"], mode=mode)
        hist = s.history()
    assert st["n_iters"] == g["converged_after"] and st["converged"] == 1
    np.testing.assert_allclose(hist, [float(r) for r in g["residuals"]], rtol=0, atol=5e-7 + 1e-12)
    assert abs(st["residual_norm"] / float(g["final_residual"]) - 1.0) <= 1e-5
    assert st["n_checks"] == len(g["residuals"])
    xo, n_o, norm_o, hist_o = oracle_run(kind, rp, col, val, b, x0)
    assert rel(x, xo) <= 1e-12
    check_hist(hist, hist_o)
    if mode == "device_loop":
        assert st["host_waits"] == 1


@pytest.mark.parametrize("kind", ["jacobi", "gauss_seidel"])
@pytest.mark.parametrize("nx,max_iters,check_length,tol", [(24, 1000, 5, 1e-8), (17, 37, 5, 1e-8),
                                                          (12, 60, 1, 0.0), (9, 300, 7, 1e-6),
                                                          (16, 4, 5, 1e-8), (8, 0, 5, 1e-8),
                                                          (72, 37, 5, 1e-8), (72, 30, 1, 0.0),
                                                          (66, 400, 7, 1e-3), (72, 3, 5, 1e-8)])
def test_loop_shapes_against_the_oracle(kind, nx, max_iters, check_length, tol):
    """Runs that converge, run out of iterations, end inside a block (a tail
    without a residual check), check every iteration, or do nothing -- on
    systems small enough for the one-CTA loop and (nx >= 66, more than 4096
    rows) on the multi-launch drivers with their graphs."""
    rp, col, val, _, _, _ = app_problem(kind, nx, gpu_perm=False)
    n = len(rp) - 1
    b = M.uniform_vector(n, 4)
    x0 = M.uniform_vector(n, 5)
    xo, n_o, norm_o, hist_o = oracle_run(kind, rp, col, val, b, x0, tol, max_iters, check_length)
    results = []
    with Solver(kind, rp, col, val) as s:
        for mode in MODES:
            x = x0.copy()
            st = s.solve(b, x, tol=tol, max_iters=max_iters, check_length=check_length, mode=mode)
            assert st["n_iters"] == n_o, mode
            assert st["n_checks"] == len(hist_o)
            check_hist(s.history(), hist_o)
            assert rel(x, xo) <= 1e-12, mode
            results.append(x)
    # every driver issues the same launches: identical results
    np.testing.assert_array_equal(results[0], results[1])
    np.testing.assert_array_equal(results[0], results[2])


@pytest.mark.parametrize("kind", ["jacobi", "gauss_seidel"])
def test_repeated_solves_reuse_the_graph(kind):
    rp, col, val, b, x0, _ = app_problem(kind, 20, gpu_perm=False)
    n = len(rp) - 1
    with Solver(kind, rp, col, val) as s:
        for seed in range(3):
            b = M.uniform_vector(n, 10 + seed)
            x = np.zeros(n)
            st = s.solve(b, x, max_iters=200)
            xo, n_o, _, _ = oracle_run(kind, rp, col, val, b, np.zeros(n), 1e-8, 200, 5)
            assert st["n_iters"] == n_o
            assert rel(x, xo) <= 1e-12


@pytest.mark.parametrize("kind", ["jacobi", "gauss_seidel"])
def test_device_arrays_and_a_caller_stream(kind):
    import torch
    rp, col, val, _, _, _ = app_problem(kind, 32, gpu_perm=False)
    n = len(rp) - 1
    b = M.uniform_vector(n, 6)
    x0 = M.uniform_vector(n, 7)
    xo, n_o, _, _ = oracle_run(kind, rp, col, val, b, x0, 1e-8, 150, 5)
    dev = torch.device("cuda")
    d_rp, d_col, d_val = (torch.from_numpy(a).to(dev) for a in (rp, col, val))
    s = Solver(kind, d_rp, d_col, d_val)
    db = torch.from_numpy(b).to(dev)
    dx = torch.from_numpy(x0).to(dev)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        st = s.solve(db, dx, max_iters=150, stream=stream.cuda_stream)
    stream.synchronize()
    assert st["n_iters"] == n_o
    assert rel(dx.cpu().numpy(), xo) <= 1e-12
    s.close()


@pytest.mark.parametrize("kind", ["jacobi", "gauss_seidel"])
def test_float32(kind):
    rp, col, val, _, _, _ = app_problem(kind, 20, gpu_perm=False)
    n = len(rp) - 1
    b = M.uniform_vector(n, 8)
    x0 = M.uniform_vector(n, 9)
    xo, _, _, _ = oracle_run(kind, rp, col, val, b, x0, 0.0, 40, 5)
    x = x0.astype(np.float32)
    with Solver(kind, rp, col, val.astype(np.float32)) as s:
        st = s.solve(b.astype(np.float32), x, tol=0.0, max_iters=40)
    assert st["n_iters"] == 40
    assert rel(x, xo) <= 1e-4


@pytest.mark.parametrize("kind", ["jacobi", "gauss_seidel"])
def test_larger_grid_fixed_iterations(kind):
    rp, col, val, _, _, _ = app_problem(kind, 256, gpu_perm=False)
    n = len(rp) - 1
    b = M.uniform_vector(n, 11)
    x0 = np.zeros(n)
    xo, n_o, norm_o, hist_o = oracle_run(kind, rp, col, val, b, x0, 0.0, 50, 10)
    x = x0.copy()
    with Solver(kind, rp, col, val) as s:
        st = s.solve(b, x, tol=0.0, max_iters=50, check_length=10)
        check_hist(s.history(), hist_o)
    assert st["n_iters"] == 50 and st["converged"] == 0
    assert rel(x, xo) <= 1e-12


def test_missing_and_zero_diagonals_are_errors():
    rp = np.array([0, 2, 3], np.int32)
    col = np.array([0, 1, 0], np.int32)  # row 1 has no diagonal entry
    val = np.array([2.0, 1.0, 1.0])
    for kind in ("jacobi", "gauss_seidel"):
        with pytest.raises(SmaxError) as e:
            Solver(kind, rp, col, val)
        assert e.value.code == -5  # SMAX_ERR_NO_DIAG
    col = np.array([0, 1, 1], np.int32)
    val = np.array([2.0, 1.0, 0.0])
    for kind in ("jacobi", "gauss_seidel"):
        with pytest.raises(SmaxError) as e:
            Solver(kind, rp, col, val)
        assert e.value.code == -4  # SMAX_ERR_ZERO_DIAG


@pytest.mark.parametrize("kind", ["jacobi", "gauss_seidel"])
def test_empty_and_one_row(kind):
    with Solver(kind, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0)) as s:
        st = s.solve(np.zeros(0), np.zeros(0))
        assert st["n_iters"] == 0 and st["converged"] == 1
    x = np.array([0.0])
    with Solver(kind, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([4.0])) as s:
        st = s.solve(np.array([2.0]), x, max_iters=10, check_length=1)
    # one iteration solves a 1x1 system exactly; the next check sees residual 0
    assert x[0] == 0.5 and st["n_iters"] == 1 and st["residual_norm"] == 0.0


def test_bad_options():
    rp, col, val = M.poisson2d_app(4)
    with Solver("jacobi", rp, col, val) as s:
        n = len(rp) - 1
        for kw in ({"check_length": 0}, {"max_iters": -1}, {"tol": float("nan")}):
            with pytest.raises(SmaxError):
                s.solve(np.ones(n), np.ones(n), **kw)
