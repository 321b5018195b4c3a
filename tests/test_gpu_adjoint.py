"""Reverse mode: the C-ABI adjoints of CRS SpMV and SpTRSV against the CPU
oracle (A^T / L^T formed on the host, reference SpMV / upper SpTRSV on them),
value updates, and the torch.autograd harness against central finite
differences (h = 1e-6, 64 random entries, seed 4) on the adjoint workloads:
y = A x with the 7-point 64^3 Laplacian and y = L^-1 b with the lower
triangle of the 5-point 512^2 Laplacian, loss = 1/2 ||y - t||^2."""
import numpy as np
import pytest

from helpers import normwise, rand_crs, tol
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
O = Oracle()


def _kernel(ktype, vt, upper=False):
    from smaxkernels_b200 import FloatType, Interface, IntType, PlatformType
    smax = Interface()
    smax.register_kernel("k", ktype, PlatformType.CUDA, IntType.INT32,
                         FloatType.FLOAT64 if vt == np.float64 else FloatType.FLOAT32)
    k = smax.kernel("k")
    if upper:
        k.set_mat_upper_triang(True)
    return smax, k


def _upper_of(rp, col, val):
    import scipy.sparse as sp
    n = len(rp) - 1
    U = sp.csr_matrix((val, col, rp), shape=(n, n)).T.tocsr()
    U.sort_indices()
    return U.indptr.astype(np.int32), U.indices.astype(np.int32), U.data.astype(val.dtype)


# ------------------------------------------------------------------ C ABI ----
@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("shape", [(3000, 2500), (2000, 2000), (1, 7)])
def test_spmv_adjoint_host(vt, shape):
    from smaxkernels_b200 import KernelType
    n, m = shape
    rp, col, val = rand_crs(n, 9, 400 + n, vt=vt, n_cols=m, empty_frac=0.1, long_rows=(m,))
    rng = np.random.default_rng(401)
    x = rng.uniform(-1, 1, m).astype(vt)
    g = rng.uniform(-1, 1, n).astype(vt)
    smax, k = _kernel(KernelType.SPMV, vt)
    y = np.zeros(n, vt)
    k.register_A(n, m, len(col), col, rp, val)
    k.register_B(m, x)
    k.register_C(n, y)
    k.run()
    dx = np.zeros(m, vt)
    dval = np.zeros(len(col), vt)
    k.adjoint(g, dx, dval)
    dx_ref, dval_ref = O.spmv_adjoint(rp, col, val, x, g, m)
    assert normwise(dx, dx_ref) <= tol(vt)
    np.testing.assert_array_equal(dval, dval_ref)  # one product per entry: exact
    # explicit x and a skipped output
    dx2 = np.zeros(m, vt)
    k.adjoint(g, dx2, None, x=x)
    np.testing.assert_array_equal(dx2, dx)
    smax.close()


@pytest.mark.parametrize("vt", [np.float64, np.float32])
@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_sptrsv_adjoint_host(vt, upper, mode):
    from smaxkernels_b200 import KernelType
    n = 4000
    rp, col, val = rand_crs(n, 7, 410, vt=vt, lower=True)
    if upper:
        rp, col, val = _upper_of(rp, col, val)
    rng = np.random.default_rng(411)
    b = rng.uniform(-1, 1, n).astype(vt)
    g = rng.uniform(-1, 1, n).astype(vt)
    smax, k = _kernel(KernelType.SPTRSV, vt, upper)
    k.set_solve_mode(mode)
    col, val = col.copy(), val.copy()
    x = np.zeros(n, vt)
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, x)
    k.register_C(n, b)
    k.run()
    # col/val now hold the diagonal-last order of the device copy
    lam = np.zeros(n, vt)
    dval = np.zeros(len(col), vt)
    k.adjoint(g, lam, dval)
    lam_ref, dval_ref = O.sptrsv_adjoint(rp, col, val, x, g, lower=not upper)
    assert normwise(lam, lam_ref) <= tol(vt)
    assert normwise(dval, dval_ref) <= tol(vt)
    # dval alone (lambda in scratch) gives the same numbers
    dval2 = np.zeros(len(col), vt)
    k.adjoint(g, None, dval2)
    np.testing.assert_array_equal(dval2, dval)
    smax.close()


def test_sptrsv_adjoint_level_scheduled():
    """The adjoint of a permuted level-scheduled solve sweeps the caller's
    levels in reverse."""
    from smaxkernels_b200 import KernelType
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace2d_5pt(60)
    n = len(rp) - 1
    smax, k = _kernel(KernelType.SPTRSV, np.float64)
    perm = np.zeros(n, np.int32)
    inv = np.zeros(n, np.int32)
    smax.utils.generate_perm(n, rp, col, perm, inv, "RS")
    prp = np.zeros(n + 1, np.int32)
    pcol = np.zeros(len(col), np.int32)
    pval = np.zeros(len(col))
    smax.utils.apply_mat_perm(n, rp, col, val, prp, pcol, pval, perm, inv)
    lrp, lcol, lval = M.lower_triangle(prp, pcol, pval)
    levels = np.array([smax.get_level_ptr_at(i) for i in range(smax.get_n_levels() + 1)], np.int32)
    k.set_mat_perm(True)
    b = np.random.default_rng(5).uniform(-1, 1, n)
    g = np.random.default_rng(6).uniform(-1, 1, n)
    x = np.zeros(n)
    lcol, lval = lcol.copy(), lval.copy()
    k.register_A(n, n, len(lcol), lcol, lrp, lval)
    k.register_B(n, x)
    k.register_C(n, b)
    k.run()
    assert normwise(x, O.sptrsv(lrp, lcol, lval, b, levels=levels)) <= 1e-12
    lam = np.zeros(n)
    dval = np.zeros(len(lcol))
    k.adjoint(g, lam, dval)
    lam_ref, dval_ref = O.sptrsv_adjoint(lrp, lcol, lval, x, g)
    assert normwise(lam, lam_ref) <= 1e-12
    assert normwise(dval, dval_ref) <= 1e-12
    smax.close()


def test_update_values_spmv_and_sptrsv():
    from smaxkernels_b200 import KernelType, SmaxError, _lib
    n = 3000
    rp, col, val = rand_crs(n, 8, 420)
    x = np.random.default_rng(421).uniform(-1, 1, n)
    smax, k = _kernel(KernelType.SPMV, np.float64)
    y = np.zeros(n)
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, x)
    k.register_C(n, y)
    k.run()
    dx0 = np.zeros(n)
    k.adjoint(np.ones(n), dx0)  # builds A^T with the old values
    val2 = (val * -1.5 + 0.25).astype(np.float64)
    k.update_A_values(val2)
    k.apply()
    k.finalize()
    assert normwise(y, O.spmv_crs(rp, col, val2, x)) <= 1e-12
    dx = np.zeros(n)
    k.adjoint(np.ones(n), dx)  # A^T values follow the update
    assert normwise(dx, O.spmv_adjoint(rp, col, val2, x, np.ones(n))[0]) <= 1e-12
    smax.close()

    rp, col, val = rand_crs(n, 6, 422, lower=True)
    b = np.random.default_rng(423).uniform(-1, 1, n)
    smax, k = _kernel(KernelType.SPTRSV, np.float64)
    col, val = col.copy(), val.copy()
    xs = np.zeros(n)
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, xs)
    k.register_C(n, b)
    k.run()
    val2 = val * 0.5
    val2[rp[1:] - 1] = 3.0 + np.arange(n) % 5  # new diagonal (last in each row)
    k.update_A_values(val2)
    k.apply()
    k.finalize()
    assert normwise(xs, O.sptrsv(rp, col, val2, b)) <= 1e-12
    bad = val2.copy()
    bad[rp[17 + 1] - 1] = 0.0
    with pytest.raises(SmaxError) as e:
        k.update_A_values(bad)
    assert e.value.code == _lib.ERR_ZERO_DIAG
    smax.close()


def test_adjoint_errors():
    from smaxkernels_b200 import KernelType, SmaxError, _lib
    rp, col, val = rand_crs(100, 4, 430)
    smax, k = _kernel(KernelType.SPMV, np.float64)
    k.register_A(100, 100, len(col), col, rp, val)
    x, y = np.zeros(100), np.zeros(100)
    k.register_B(100, x)
    k.register_C(100, y)
    with pytest.raises(SmaxError) as e:  # not initialized
        k.adjoint(np.ones(100), np.zeros(100))
    assert e.value.code == _lib.ERR_STATE
    smax.close()
    smax, k = _kernel(KernelType.SPMM, np.float64)
    k.register_A(100, 100, len(col), col, rp, val)
    X, Y = np.zeros(400), np.zeros(400)
    k.register_B(100, 4, X)
    k.register_C(100, 4, Y)
    k.run()
    with pytest.raises(SmaxError) as e:
        k.adjoint(np.ones(400), np.zeros(400))
    assert e.value.code == _lib.ERR_UNSUPPORTED
    smax.close()


# --------------------------------------------------------------- autograd ----
def _fd_check(fwd, params, t, entries_of, h=1e-6, rel=1e-6):
    """Central differences of loss = 1/2||fwd() - t||^2 for the given entries of
    each parameter, through the stable form
    (L+ - L-) = sum 1/2 (y+ - y-)(y+ + y- - 2t)."""
    import torch
    worst = 0.0
    for p, idx in entries_of:
        for i in idx:
            old = p[i].item()
            p[i] = old + h
            yp = fwd().detach()
            p[i] = old - h
            ym = fwd().detach()
            p[i] = old
            fd = float((0.5 * (yp - ym) * (yp + ym - 2 * t)).sum()) / (2 * h)
            ad = float(p.grad[i])
            err = abs(fd - ad) / max(1.0, abs(ad))
            worst = max(worst, err)
            assert err <= rel, (i, fd, ad)
    return worst


def test_autograd_spmv_laplace64_fd_and_oracle():
    import torch
    from smaxkernels_b200 import matrices as M
    from smaxkernels_b200.autograd import SparsePattern, spmv
    rp, col, val = M.laplace3d_7pt(64)
    n = len(rp) - 1
    rng = np.random.default_rng(4)
    x0 = rng.uniform(-1, 1, n)
    t0 = rng.uniform(-1, 1, n)
    A = SparsePattern(rp, col, kind="spmv")
    v = torch.tensor(val, device="cuda", requires_grad=True)
    x = torch.tensor(x0, device="cuda", requires_grad=True)
    t = torch.tensor(t0, device="cuda")
    y = spmv(A, v, x)
    loss = 0.5 * ((y - t) ** 2).sum()
    loss.backward()
    g = (y - t).detach().cpu().numpy()
    dx_ref, dval_ref = O.spmv_adjoint(rp, col, val, x0, g)
    assert normwise(x.grad.cpu().numpy(), dx_ref) <= 1e-12
    assert normwise(v.grad.cpu().numpy(), dval_ref) <= 1e-12
    pick = np.random.default_rng(4)
    idx_v = pick.choice(len(col), 64, replace=False)
    idx_x = pick.choice(n, 64, replace=False)
    with torch.no_grad():
        _fd_check(lambda: spmv(A, v, x), [v, x], t, [(v, idx_v), (x, idx_x)])


def test_autograd_sptrsv_laplace512_fd_and_oracle():
    import torch
    from smaxkernels_b200 import matrices as M
    from smaxkernels_b200.autograd import SparsePattern, sptrsv
    rp, col, val = M.lower_triangle(*M.laplace2d_5pt(512))
    n = len(rp) - 1
    rng = np.random.default_rng(4)
    b0 = rng.uniform(-1, 1, n)
    t0 = rng.uniform(-1, 1, n)
    L = SparsePattern(rp, col, kind="sptrsv")
    v = torch.tensor(val, device="cuda", requires_grad=True)
    b = torch.tensor(b0, device="cuda", requires_grad=True)
    t = torch.tensor(t0, device="cuda")
    x = sptrsv(L, v, b)
    assert normwise(x.detach().cpu().numpy(), O.sptrsv(rp, col, val, b0)) <= 1e-12
    loss = 0.5 * ((x - t) ** 2).sum()
    loss.backward()
    g = (x - t).detach().cpu().numpy()
    lam_ref, dval_ref = O.sptrsv_adjoint(rp, col, val, x.detach().cpu().numpy(), g)
    assert normwise(b.grad.cpu().numpy(), lam_ref) <= 1e-12
    assert normwise(v.grad.cpu().numpy(), dval_ref) <= 1e-12
    pick = np.random.default_rng(4)
    idx_v = pick.choice(len(col), 64, replace=False)
    idx_b = pick.choice(n, 64, replace=False)
    with torch.no_grad():
        _fd_check(lambda: sptrsv(L, v, b), [v, b], t, [(v, idx_v), (b, idx_b)])


def test_autograd_sptrsv_diagonal_first_rows_and_float32():
    """Rows whose diagonal is not last in the caller's order: gradients come
    back in the caller's entry order."""
    import torch
    from smaxkernels_b200.autograd import SparsePattern, sptrsv
    n = 500
    rp, col, val = rand_crs(n, 5, 440, lower=True)
    col2, val2 = col.copy(), val.copy()
    for r in range(n):
        s, e = rp[r], rp[r + 1]
        col2[s:e] = np.roll(col[s:e], 1)
        val2[s:e] = np.roll(val[s:e], 1)
    for dt, tl in ((torch.float64, 1e-12), (torch.float32, 1e-5)):
        L = SparsePattern(rp, col2, kind="sptrsv", dtype=dt)
        v = torch.tensor(val2, device="cuda", dtype=dt, requires_grad=True)
        b = torch.tensor(np.linspace(-1, 1, n), device="cuda", dtype=dt, requires_grad=True)
        x = sptrsv(L, v, b)
        x.sum().backward()
        xd = x.detach().double().cpu().numpy()
        lam_ref, dval_ref = O.sptrsv_adjoint(rp, col2, val2, xd, np.ones(n))
        assert normwise(b.grad.double().cpu().numpy(), lam_ref) <= tl
        assert normwise(v.grad.double().cpu().numpy(), dval_ref) <= tl


def test_autograd_adjoint_time_budget():
    """Backward (adjoint) time of the SpMV workload stays within 2x the forward."""
    import torch
    from smaxkernels_b200 import matrices as M
    from smaxkernels_b200.autograd import SparsePattern
    rp, col, val = M.laplace3d_7pt(64)
    n = len(rp) - 1
    A = SparsePattern(rp, col, kind="spmv")
    v = torch.tensor(val, device="cuda")
    x = torch.rand(n, device="cuda", dtype=torch.float64)
    g = torch.rand(n, device="cuda", dtype=torch.float64)
    A.forward(v, x)
    A.backward(v, x, g, True, True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st = torch.cuda.current_stream()

    def timed(f, reps=50):
        f()
        e0.record(st)
        for _ in range(reps):
            f()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    tf = timed(lambda: A.k.apply())
    tb = timed(lambda: A.k.adjoint(A._g, A._din, A._dval, x=x))
    assert tb <= 2.5 * tf + 0.02, (tf, tb)
