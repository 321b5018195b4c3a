"""Pins the oracle's restatement of the reference's Matrix Market reader
(Oracle.read_mtx) against the reference's own reader, COOMatrix::read_from_mtx
+ convert_coo_to_crs compiled from examples/matrix_structs.hpp
(Reference.read_mtx): identical arrays for every accepted file form, and
both refuse the same files."""
import numpy as np
import pytest

import mtx_files
from oracle.oracle import Oracle, Reference, reference_available

needs_ref = pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")


@needs_ref
def test_oracle_reader_equals_the_reference_reader(tmp_path):
    R = Reference()
    for name, path in mtx_files.accepted(str(tmp_path)).items():
        got = Oracle.read_mtx(path)
        ref = R.read_mtx(path)
        assert got[:3] == ref[:3], name
        for a, b in zip(got[3:], ref[3:]):
            np.testing.assert_array_equal(a, b, err_msg=name)
        # -0.0 is kept as written
        assert np.array_equal(np.signbit(got[5]), np.signbit(ref[5])), name


@needs_ref
def test_both_refuse_the_same_files(tmp_path):
    R = Reference()
    for name, path in mtx_files.rejected(str(tmp_path)).items():
        with pytest.raises(ValueError):
            Oracle.read_mtx(path)
        with pytest.raises(RuntimeError):
            R.read_mtx(path)


def test_the_oracle_refuses_a_truncated_file(tmp_path):
    with pytest.raises(ValueError):
        Oracle.read_mtx(mtx_files.truncated(str(tmp_path)))


def test_stable_row_order_keeps_the_file_order(tmp_path):
    p = mtx_files.write(str(tmp_path / "t.mtx"), "%%MatrixMarket matrix coordinate real general", (3, 3, 5),
                        [("2", "3", "1"), ("1", "2", "2"), ("2", "1", "3"), ("1", "1", "4"), ("3", "3", "5")])
    n, m, z, rp, col, val = Oracle.read_mtx(p)
    assert rp.tolist() == [0, 2, 4, 5]
    assert col.tolist() == [1, 0, 2, 0, 2] and val.tolist() == [2.0, 4.0, 1.0, 3.0, 5.0]
