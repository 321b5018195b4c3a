"""Typed views of the golden fixtures extracted from the reference's unit tests.

Each helper turns one examples/tests/*.hpp record of tests/golden/reference_tests.json
into numpy arrays plus the expected outputs, so the same case can be replayed
against the oracle (CPU) and against the CUDA kernels (GPU).
"""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_REF = None


def ref_tests() -> dict:
    global _REF
    if _REF is None:
        with open(os.path.join(HERE, "golden", "reference_tests.json")) as f:
            _REF = json.load(f)
    return _REF


def laplace() -> dict:
    with open(os.path.join(HERE, "golden", "bcrs_laplace.json")) as f:
        return json.load(f)


def _vt(rec, default="double"):
    t = rec["types"].get("VT")
    if t is None:
        tp = next(iter(rec["ctors"].values()))["tparams"]
        t = tp.split(",")[1] if "," in tp else default
    return np.float32 if t == "float" else np.float64


def almost_equal(a, b, dtype) -> bool:
    """The reference's comparison rule (examples/tests/tests_common.hpp:9-35):
    |a-b| <= abs_eps, or |a-b| <= 4*eps*max(|a|,|b|); abs_eps 1e-14 (double),
    1e-7 (float)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if np.dtype(dtype) == np.float32:
        abs_eps, rel = 1e-7, 4 * float(np.finfo(np.float32).eps)
    else:
        abs_eps, rel = 1e-14, 4 * float(np.finfo(np.float64).eps)
    d = np.abs(a - b)
    return bool(np.all((d <= abs_eps) | (d <= rel * np.maximum(np.abs(a), np.abs(b)))))


def crs(rec, prefix):
    a = rec["arrays"]
    vt = _vt(rec)
    rp = np.array(a[prefix + "->row_ptr"], dtype=np.int32)
    col = np.array(a[prefix + "->col"], dtype=np.int32)
    val = np.array(a[prefix + "->val"], dtype=vt) if prefix + "->val" in a else np.ones(len(col), vt)
    return rp, col, val


def spmv_case(name="spmv_test"):
    r = ref_tests()[name]
    rp, col, val = crs(r, "A")
    n_cols = r["ctors"]["A"]["args"][1]
    x = np.full(n_cols, r["fills"]["x"], dtype=val.dtype)
    return dict(row_ptr=rp, col=col, val=val, x=x, y=np.array(r["arrays"]["y_expected"], val.dtype))


SCS_TESTS = ["spmv_scs_1_1_test_1", "spmv_scs_1_1_test_2", "spmv_scs_1_4_test_1", "spmv_scs_2_1_test_1",
             "spmv_scs_2_1_test_2", "spmv_scs_2_4_test_1", "spmv_scs_4_1_test_1", "spmv_scs_4_1_test_2",
             "spmv_scs_4_4_test_1"]


def scs_case(name):
    r = ref_tests()[name]
    rp, col, val = crs(r, "A_crs")
    C_, sigma = r["ctors"]["A_scs"]["args"][:2]
    a, f = r["arrays"], r["fields"]
    exp = dict(C=C_, sigma=sigma, n_rows=f["A_scs_exp->n_rows"], n_rows_padded=f["A_scs_exp->n_rows_padded"],
               n_cols=f["A_scs_exp->n_cols"], n_chunks=f["A_scs_exp->n_chunks"],
               n_elements=f["A_scs_exp->n_elements"], nnz=f.get("A_scs_exp->nnz", len(col)),
               chunk_ptr=np.array(a["A_scs_exp->chunk_ptr"], np.int32),
               chunk_lengths=np.array(a["A_scs_exp->chunk_lengths"], np.int32),
               col=np.array(a["A_scs_exp->col"], np.int32), val=np.array(a["A_scs_exp->val"], val.dtype),
               perm=np.array(a["A_scs_exp->perm"], np.int32))
    return dict(row_ptr=rp, col=col, val=val, C=C_, sigma=sigma, expected=exp)


BCRS_CONV_TESTS = ["spmv_bcrs_1_1_test_1", "spmv_bcrs_1_1_test_2"]


def bcrs_conv_case(name):
    r = ref_tests()[name]
    rp, col, val = crs(r, "A_crs")
    c, a = r["consts"], r["arrays"]
    exp_args = r["ctors"]["A_bcrs_exp"]["args"]
    return dict(row_ptr=rp, col=col, val=val, n_cols=r["fields"]["A_crs->n_cols"],
                bh=c["target_b_height"], bw=c["target_b_width"], hpad=c["target_height_pad"],
                wpad=c["target_width_pad"], col_major=bool(c["use_blocked_column_major"]),
                expected=dict(n_rows=exp_args[0], n_cols=exp_args[1], n_blocks=exp_args[2],
                              row_ptr=np.array(a["A_bcrs_exp->row_ptr"], np.int32),
                              col=np.array(a["A_bcrs_exp->col"], np.int32),
                              val=np.array(a["A_bcrs_exp->val"], val.dtype)))


def bcrs_spmv_case(name="spmv_bcrs_1_1_test_3"):
    r = ref_tests()[name]
    a = r["arrays"]
    nr, nc, nb, bh, bw, hp, wp = r["ctors"]["A_bcrs"]["args"]
    x = np.zeros(nc * wp)
    x[: nc * bw] = r["fills"]["x"]
    return dict(n_rows=nr, n_cols=nc, n_blocks=nb, b_height=bh, b_width=bw, height_pad=hp, width_pad=wp,
                row_ptr=np.array(a["A_bcrs->row_ptr"], np.int32), col=np.array(a["A_bcrs->col"], np.int32),
                val=np.array(a["A_bcrs->val"], np.float64), col_major=bool(r["consts"]["block_column_major"]),
                x=x, y=np.array(a["y_expected"], np.float64))


def spmm_case(name):
    r = ref_tests()[name]
    rp, col, val = crs(r, "A")
    k = r["consts"]["n_vectors"]
    n_cols = r["ctors"]["A"]["args"][1]
    row_major = ["set_vec_row_major", "true"] in r["flags"]
    X = np.full(n_cols * k, r["fills"]["X"], dtype=val.dtype)
    return dict(row_ptr=rp, col=col, val=val, k=k, X=X, row_major=row_major,
                Y=np.array(r["arrays"]["Y_expected"], val.dtype))


def spgemm_case(name):
    r = ref_tests()[name]
    a = r["arrays"]
    A = crs(r, "A")
    B = crs(r, "B") if "B->row_ptr" in a else A
    itype = r["types"].get("IT", "int")
    return dict(A=A, B=B, b_n_cols=r["ctors"]["A"]["args"][1], itype=itype,
                C=(np.array(a["C_exp->row_ptr"], np.int32), np.array(a["C_exp->col"], np.int32),
                   np.array(a["C_exp->val"], A[2].dtype)))


def sptrsv_case(name="sptrsv_test"):
    r = ref_tests()[name]
    rp, col, val = crs(r, "A")
    n = len(rp) - 1
    b = np.full(n, r["fills"]["b"], dtype=val.dtype)
    return dict(row_ptr=rp, col=col, val=val, b=b, x=np.array(r["arrays"]["x_expected"], val.dtype))


def sptrsm_case(name):
    r = ref_tests()[name]
    rp, col, val = crs(r, "A")
    n = len(rp) - 1
    k = r["consts"]["n_vectors"]
    row_major = ["set_vec_row_major", "true"] in r["flags"]
    B = np.full(n * k, r["fills"]["B"], dtype=val.dtype)
    return dict(row_ptr=rp, col=col, val=val, k=k, B=B, row_major=row_major,
                X=np.array(r["arrays"]["X_expected"], val.dtype))


def perm_case(name):
    r = ref_tests()[name]
    rp, col, val = crs(r, "A")
    a = r["arrays"]
    return dict(row_ptr=rp, col=col, val=val, n_levels=r["consts"]["expected_max_level"],
                lvl_ptr=np.array(a["expected_levels"], np.int32),
                perm_bfs=np.array(a["expected_perm_bfs"], np.int32),
                perm_rs=np.array(a["expected_perm_rs"], np.int32),
                val_bfs=np.array(a["expected_val_bfs"], np.float64),
                val_rs=np.array(a["expected_val_rs"], np.float64))


def symmetric_case(name):
    r = ref_tests()[name]
    a = r["arrays"]
    return dict(row_ptr=np.array(a["A->row_ptr"], np.int32), col=np.array(a["A->col"], np.int32),
                sym_row_ptr=np.array(a["A_sym_exp->row_ptr"], np.int32),
                sym_col=np.array(a["A_sym_exp->col"], np.int32))


def sort_rows(row_ptr, col):
    """examples/examples_common.hpp:425 sort_crs_rows_by_col (pattern only)."""
    out = np.array(col, copy=True)
    for r in range(len(row_ptr) - 1):
        out[row_ptr[r]:row_ptr[r + 1]] = np.sort(out[row_ptr[r]:row_ptr[r + 1]])
    return out
