"""The cuSPARSE comparison (bench.py --workload cusparse) compares like with
like: on the same device arrays, cuSPARSE called through torch.sparse with
the library's default algorithms gives the same results as this platform's
kernels -- CSR SpMV, BSR 4x4 SpMV, CSR SpMM against a row-major block, and
SpGEMM's pattern up to column order (cuSPARSE sorts each row's columns, the
reference keeps first-touch order).  Small cases of the benchmark's matrices."""
import numpy as np
import pytest

from helpers import normwise

pytestmark = pytest.mark.gpu


def _csr(torch, rp, col, val, n_cols):
    return torch.sparse_csr_tensor(torch.from_numpy(rp.astype(np.int32)).cuda(),
                                   torch.from_numpy(col.astype(np.int32)).cuda(), torch.from_numpy(val).cuda(),
                                   size=(len(rp) - 1, n_cols))


@pytest.mark.parametrize("case", ["lognormal_65536", "laplace3d_24"])
def test_csr_spmv_matches_cusparse(case):
    import torch
    from helpers import gpu_spmv
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.lognormal_random(1 << 16, seed=1) if case.startswith("lognormal") else M.laplace3d_7pt(24)
    n = len(rp) - 1
    x = M.uniform_vector(n, 100)
    y_lib = torch.mv(_csr(torch, rp, col, val, n), torch.from_numpy(x).cuda()).cpu().numpy()
    assert normwise(gpu_spmv(rp, col, val, x), y_lib) <= 1e-12


def test_bsr4x4_spmv_matches_cusparse():
    import torch
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace3d_7pt(24)
    n = len(rp) - 1
    x = M.uniform_vector(n, 100)
    smax = Interface()
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    k.set_mat_bcrs(True)
    bc = smax.utils.convert_crs_to_bcrs(n, n, len(col), col, rp, val, 4, 4, 4, 4, False)
    y = np.zeros(n)
    k.register_A(bc["n_rows"], bc["n_cols"], bc["n_blocks"], 4, 4, 4, 4, bc["col"], bc["row_ptr"], bc["val"])
    k.register_B(n, x)
    k.register_C(n, y)
    k.run()
    smax.close()
    nb = bc["n_blocks"]
    Ab = torch.sparse_bsr_tensor(torch.from_numpy(bc["row_ptr"]).cuda(), torch.from_numpy(bc["col"]).cuda(),
                                 torch.from_numpy(bc["val"]).cuda().view(nb, 4, 4), size=(n, n))
    y_lib = torch.mv(Ab, torch.from_numpy(x).cuda()).cpu().numpy()
    assert normwise(y, y_lib) <= 1e-12


def test_csr_spmm_row_major_matches_cusparse():
    import torch
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.stencil27(24)
    n, kv = len(rp) - 1, 16
    X = np.random.default_rng(2).uniform(-1, 1, n * kv)
    smax = Interface()
    smax.register_kernel("k", KernelType.SPMM, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    Y = np.zeros(n * kv)
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, kv, X)
    k.register_C(n, kv, Y)
    k.set_vec_row_major(True)
    k.run()
    smax.close()
    Y_lib = torch.mm(_csr(torch, rp, col, val, n), torch.from_numpy(X).cuda().view(n, kv)).reshape(-1).cpu().numpy()
    assert normwise(Y, Y_lib) <= 1e-12


def test_spgemm_pattern_matches_cusparse_up_to_column_order():
    import torch
    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace3d_7pt(20)
    n = len(rp) - 1
    smax = Interface()
    smax.register_kernel("g", KernelType.SPGEMM, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("g")
    k.register_A(n, n, len(col), col, rp, val)
    k.register_B(n, n, len(col), col, rp, val)
    k.register_C()
    k.run()
    _, _, nnz, crp, ccol, cval = k.result()
    smax.close()
    A = _csr(torch, rp, col, val, n)
    C = torch.mm(A, A).to_sparse_csr()
    lrp, lcol, lval = (t.cpu().numpy() for t in (C.crow_indices(), C.col_indices(), C.values()))
    np.testing.assert_array_equal(crp, lrp)
    for r in range(n):  # same columns and values per row; cuSPARSE sorts them
        a, b = crp[r], crp[r + 1]
        o = np.argsort(ccol[a:b], kind="stable")
        np.testing.assert_array_equal(ccol[a:b][o], lcol[a:b])
        assert normwise(cval[a:b][o], lval[a:b]) <= 1e-12
