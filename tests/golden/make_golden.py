"""Regenerates the golden fixtures in tests/golden/ from the reference checkout.

Usage (from the repository root, where the reference checkout exists):

    python tests/golden/make_golden.py [--ref-root PATH]

1. reference_tests.json -- for every known-answer unit test of the hot path in
   the reference (examples/tests/*.hpp), the literal data the test holds: its
   brace-initialised arrays (inputs and expected outputs), constructor
   arguments, scalar field assignments, integer/bool constants, uniform fill
   values (``x[i] = 1.0``), type aliases and flag setter calls.  Nothing is
   retyped by hand; the values are parsed from the test sources as text.

3. solver_apps.json -- the printed output of the reference's two iterative-
   solver applications, examples/applications/{jacobi,gauss_seidel}, built
   unmodified by ``make -C oracle apps`` (oracle/_ref/jacobi, gauss_seidel)
   and run with one OpenMP thread (the BFS permutation the Jacobi program
   prints is thread-order dependent): the permutation, the residual printed
   every CHECK_LENGTH iterations ("%f"), the iteration count and the final
   residual (6 significant digits).

2. bcrs_laplace.json -- examples/tests/spmv_bcrs_laplace_test.hpp builds its
   input in code (a 16x16 tridiagonal 2/-1 matrix, x_i = 1/((i+3)%23+1),
   4x8 blocks in both in-block orders).  The same construction is restated
   below and the expected outputs are produced by the reference itself
   (oracle/_ref/libsmax_ref.so, built by ``make -C oracle ref``).

The fixtures are committed; tests read only the JSON files and never the
reference checkout.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

TESTS = [
    "spmv_test", "spmv_bcrs_1_1_test_1", "spmv_bcrs_1_1_test_2", "spmv_bcrs_1_1_test_3",
    "spmv_scs_1_1_test_1", "spmv_scs_1_1_test_2", "spmv_scs_1_4_test_1", "spmv_scs_2_1_test_1",
    "spmv_scs_2_1_test_2", "spmv_scs_2_4_test_1", "spmv_scs_4_1_test_1", "spmv_scs_4_1_test_2",
    "spmv_scs_4_4_test_1", "spmm_test", "spmm_rowmaj_test", "spgemmAA_test", "spgemmAB_test",
    "sptrsv_test", "sptrsm_test", "sptrsm_rowmaj_test", "perm_test_1", "perm_test_2",
    "build_symmetric_crs_1", "build_symmetric_crs_2", "build_symmetric_crs_3",
]

_NUM = re.compile(r"^-?(\d+\.?\d*|\.\d+)([eE][-+]?\d+)?[fF]?$")


def _num(tok: str):
    tok = tok.strip()
    if not _NUM.match(tok):
        return tok
    t = tok.rstrip("fF")
    if re.match(r"^-?\d+$", t):
        return int(t)
    return float(t)


def _strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def parse_test(path: str) -> dict:
    src = _strip_comments(open(path).read())
    out = {"arrays": {}, "ctors": {}, "fields": {}, "consts": {}, "fills": {}, "types": {}, "flags": []}
    for m in re.finditer(r"([\w>\-]+)\s*=\s*new\s+[\w:]+\s*\[[^\]]*\]\s*\{([^}]*)\}", src, flags=re.S):
        toks = [t for t in m.group(2).replace("\n", " ").split(",") if t.strip()]
        out["arrays"][m.group(1)] = [_num(t) for t in toks]
    for m in re.finditer(r"(\w+)\s*=\s*new\s+(CRSMatrix|SCSMatrix|BCRSMatrix)\s*<([^>]*)>\s*\(([^)]*)\)", src,
                         flags=re.S):
        args = [a for a in m.group(4).replace("\n", " ").split(",") if a.strip()]
        out["ctors"][m.group(1)] = {"type": m.group(2), "tparams": m.group(3).replace(" ", ""),
                                    "args": [_num(a) for a in args]}
    for m in re.finditer(r"(\w+->\w+)\s*=\s*(-?[0-9][0-9.eE+\-]*)\s*;", src):
        out["fields"][m.group(1)] = _num(m.group(2))
    for m in re.finditer(r"(?:const\s+)?(?:int|bool)\s+(\w+)\s*=\s*(\w+)\s*;", src):
        v = m.group(2)
        out["consts"][m.group(1)] = {"true": True, "false": False}.get(v, _num(v))
    for m in re.finditer(r"(\w+)\[i\]\s*=\s*(-?[0-9.]+)\s*;", src):
        out["fills"][m.group(1)] = _num(m.group(2))
    for m in re.finditer(r"using\s+(IT|VT)\s*=\s*([\w:]+)\s*;", src):
        out["types"][m.group(1)] = m.group(2)
    for m in re.finditer(r"->\s*(set_\w+)\(([^)]*)\)", src):
        out["flags"].append([m.group(1), m.group(2).strip()])
    for m in re.finditer(r"register_kernel\(([^;]*)\);", src, flags=re.S):
        out.setdefault("register_kernel", []).append(" ".join(m.group(1).split()))
    return out


def laplace_fixture() -> dict:
    """Input construction of spmv_bcrs_laplace_test.hpp (mat_size = 16) and the
    reference's own outputs for it."""
    import numpy as np
    sys.path.insert(0, REPO)
    from oracle.oracle import Reference

    n = 16
    rows, cols, vals = [], [], []
    for i in range(n):
        for j, v in ((i - 1, -1.0), (i, 2.0), (i + 1, -1.0)):
            if 0 <= j < n:
                rows.append(i)
                cols.append(j)
                vals.append(v)
    row_ptr = np.zeros(n + 1, dtype=np.int32)
    np.add.at(row_ptr, np.array(rows) + 1, 1)
    row_ptr = np.cumsum(row_ptr).astype(np.int32)
    col = np.array(cols, dtype=np.int32)
    val = np.array(vals, dtype=np.float64)
    x = np.array([1.0 / float((i + 3) % 23 + 1) for i in range(n)])
    R = Reference()
    y = R.spmv_crs(row_ptr, col, val, x)
    fx = {"n": n, "row_ptr": row_ptr.tolist(), "col": col.tolist(), "val": val.tolist(), "x": x.tolist(),
          "y_crs": y.tolist(), "bh": 4, "bw": 8, "hpad": 4, "wpad": 8, "bcrs": {}}
    for cm in (True, False):
        b = R.bcrs(row_ptr, col, val, n, 4, 8, 4, 8, cm)
        yb = R.spmv_bcrs(b, x, cm)
        fx["bcrs"]["col_major" if cm else "row_major"] = {
            "n_rows": b["n_rows"], "n_cols": b["n_cols"], "n_blocks": b["n_blocks"],
            "row_ptr": b["row_ptr"].tolist(), "col": b["col"].tolist(), "val": b["val"].tolist(),
            "y": yb.tolist()}
    return fx


def solver_apps_fixture() -> dict:
    import subprocess
    out = {}
    env = dict(os.environ, OMP_NUM_THREADS="1")
    for app in ("jacobi", "gauss_seidel"):
        exe = os.path.join(REPO, "oracle", "_ref", app)
        run = subprocess.run([exe], capture_output=True, text=True, env=env, cwd=os.path.join(REPO, "oracle", "_ref"),
                             check=True)
        rec = {"program": f"examples/applications/{app}/{app}.cpp", "domain_size": 10, "tol": 1e-8,
               "max_iters": 1000, "check_length": 5, "iters": [], "residuals": []}
        for line in run.stdout.splitlines():
            m = re.match(r"iter: (\d+), residual_norm = (\S+)", line)
            if m:
                rec["iters"].append(int(m.group(1)))
                rec["residuals"].append(m.group(2))
            m = re.match(r"Using permutation vector: \[(.*)\]", line)
            if m:
                rec["perm"] = [int(t) for t in m.group(1).split(",")]
            m = re.match(r".* solver converged after (\d+) iterations", line)
            if m:
                rec["converged_after"] = int(m.group(1))
            m = re.match(r"Final residual norm: (\S+)", line)
            if m:
                rec["final_residual"] = m.group(1)
        out[app] = rec
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=os.environ.get("SMAX_REF_ROOT", "/root/reference"),
                    help="the reference checkout (default: $SMAX_REF_ROOT, else /root/reference)")
    a = ap.parse_args()
    tdir = os.path.join(a.ref_root, "examples", "tests")
    data = {}
    for t in TESTS:
        data[t] = parse_test(os.path.join(tdir, t + ".hpp"))
        data[t]["source"] = f"examples/tests/{t}.hpp"
    with open(os.path.join(HERE, "reference_tests.json"), "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    with open(os.path.join(HERE, "bcrs_laplace.json"), "w") as f:
        json.dump(laplace_fixture(), f, indent=1)
    with open(os.path.join(HERE, "solver_apps.json"), "w") as f:
        json.dump(solver_apps_fixture(), f, indent=1)
    print("wrote", len(data), "test fixtures")


if __name__ == "__main__":
    main()
