"""Matrix Market ingestion (smax_utils_read_mtx, smax_utils_convert_coo_to_crs)
against the oracle's restatement of the reference's reader: bit-exact CRS
arrays for every accepted form, the reference's refusals as statuses, and
the multi-threaded parse of large files (including an entry split over two
lines across a slice cut, which falls back to one slice)."""
import numpy as np
import pytest

import mtx_files
from oracle.oracle import Oracle
from smaxkernels_b200 import Interface
from smaxkernels_b200._lib import SmaxError
from smaxkernels_b200 import matrices as M

pytestmark = pytest.mark.gpu


def same(got, ref, dtype=np.float64):
    assert tuple(got[:3]) == tuple(ref[:3])
    np.testing.assert_array_equal(got[3], ref[3])
    np.testing.assert_array_equal(got[4], ref[4])
    np.testing.assert_array_equal(got[5], ref[5].astype(dtype))
    assert np.array_equal(np.signbit(got[5]), np.signbit(ref[5].astype(dtype)))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_every_accepted_form(tmp_path, dtype):
    smax = Interface()
    for name, path in mtx_files.accepted(str(tmp_path)).items():
        same(smax.utils.read_mtx(path, dtype), Oracle.read_mtx(path), dtype)
    smax.close()


def test_refusals(tmp_path):
    smax = Interface()
    codes = {"complex": -10, "array": -10, "hermitian": -10, "skew": -10, "no_banner": -1}
    for name, path in mtx_files.rejected(str(tmp_path)).items():
        with pytest.raises(SmaxError) as e:
            smax.utils.read_mtx(path)
        assert e.value.code == codes[name], name
    with pytest.raises(SmaxError) as e:
        smax.utils.read_mtx(mtx_files.truncated(str(tmp_path)))
    assert e.value.code == -1
    for entries, code in (([("4", "1", "1.0")], -1), ([("1", "4", "1.0")], -8), ([("0", "1", "1.0")], -1),
                          ([("1", "x", "1.0")], -1), ([("1", "1", "1.0z")], -1)):
        p = mtx_files.write(str(tmp_path / "bad.mtx"), "%%MatrixMarket matrix coordinate real general", (3, 3, 1),
                            entries)
        with pytest.raises(SmaxError) as e:
            smax.utils.read_mtx(p)
        assert e.value.code == code, entries
    with pytest.raises(SmaxError):
        smax.utils.read_mtx(str(tmp_path / "does_not_exist.mtx"))
    smax.close()


def _big_file(path, split_some=False):
    rp, col, val = M.laplace3d_7pt(40)
    n = len(rp) - 1
    row_of = np.repeat(np.arange(n), np.diff(rp))
    rng = np.random.default_rng(3)
    order = rng.permutation(len(col))
    v = rng.uniform(-1, 1, len(col))
    lines = []
    for i, k in enumerate(order):
        if split_some and i % 997 == 0:
            lines.append(f"{row_of[k] + 1} {col[k] + 1}\n{float(v[k])!r}")
        else:
            lines.append(f"{row_of[k] + 1} {col[k] + 1} {float(v[k])!r}")
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{n} {n} {len(col)}\n")
        f.write("\n".join(lines) + "\n")
    return path


@pytest.mark.parametrize("split", [False, True])
def test_large_file_parallel_parse(tmp_path, split):
    p = _big_file(str(tmp_path / "big.mtx"), split)
    smax = Interface()
    same(smax.utils.read_mtx(p), Oracle.read_mtx(p))
    smax.close()


def test_coo_to_crs_host_and_device(tmp_path):
    import torch
    rng = np.random.default_rng(5)
    n, m, z = 300, 200, 5000
    I = rng.integers(0, n, z).astype(np.int32)
    J = rng.integers(0, m, z).astype(np.int32)
    V = rng.uniform(-1, 1, z)
    order = np.argsort(I, kind="stable")
    rp = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(I, minlength=n), out=rp[1:])
    smax = Interface()
    got = smax.utils.convert_coo_to_crs(n, m, I, J, V)
    np.testing.assert_array_equal(got[0], rp)
    np.testing.assert_array_equal(got[1], J[order])
    np.testing.assert_array_equal(got[2], V[order])
    # device arrays go through the same call
    from smaxkernels_b200.interface import _ptr, _take
    import ctypes as C
    from smaxkernels_b200._lib import check, lib
    dI, dJ, dV = (torch.from_numpy(a).cuda() for a in (I, J, V))
    ptrs = [C.c_void_p() for _ in range(3)]
    check(lib.smax_utils_convert_coo_to_crs(1, n, m, z, _ptr(dI), _ptr(dJ), _ptr(dV), *[C.byref(p) for p in ptrs]))
    np.testing.assert_array_equal(_take(ptrs[0].value, n + 1, np.int32), rp)
    np.testing.assert_array_equal(_take(ptrs[1].value, z, np.int32), J[order])
    np.testing.assert_array_equal(_take(ptrs[2].value, z, np.float64), V[order])
    smax.close()


def test_read_matrix_runs_through_spmv(tmp_path):
    """A file read by the platform feeds a kernel directly."""
    from smaxkernels_b200 import FloatType, IntType, KernelType, PlatformType
    path = mtx_files.accepted(str(tmp_path))["symmetric_real"]
    smax = Interface()
    n, m, z, rp, col, val = smax.utils.read_mtx(path)
    x = M.uniform_vector(m, 1)
    y = np.zeros(n)
    smax.register_kernel("k", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64)
    k = smax.kernel("k")
    k.register_A(n, m, z, col, rp, val)
    k.register_B(m, x)
    k.register_C(n, y)
    k.run()
    yo = Oracle().spmv_crs(rp, col, val, x)
    assert np.linalg.norm(y - yo) <= 1e-12 * np.linalg.norm(yo)
    smax.close()
