"""Matrix Market files for the ingestion tests, written into a directory:
every form the reference's reader accepts (real / integer / pattern values,
general / symmetric storage), with comment and blank lines, CRLF line ends,
entries in scrambled order with duplicates, and files it rejects."""
import os

import numpy as np


def _entries(rng, n_rows, n_cols, nnz, lower=False):
    I = rng.integers(0, n_rows, nnz)
    J = rng.integers(0, n_cols, nnz)
    if lower:
        I, J = np.maximum(I, J), np.minimum(I, J)
    return I, J


def write(path, banner, size, entries, comments=("% made for the ingestion tests",), eol="\n", blank=False):
    with open(path, "w", newline="") as f:
        f.write(banner + eol)
        for c in comments:
            f.write(c + eol)
        if blank:
            f.write(eol)
        f.write(" ".join(str(s) for s in size) + eol)
        for e in entries:
            f.write(" ".join(e) + eol)
    return path


def accepted(d, seed=0):
    """{name: path} of files the reference reads."""
    rng = np.random.default_rng(seed)
    out = {}
    I, J = _entries(rng, 37, 29, 300)
    V = rng.uniform(-1, 1, 300)
    V[::17] = -0.0
    out["general_real"] = write(os.path.join(d, "general_real.mtx"), "%%MatrixMarket matrix coordinate real general",
                                (37, 29, 300), [(str(i + 1), str(j + 1), repr(float(v))) for i, j, v in zip(I, J, V)])
    I, J = _entries(rng, 50, 50, 400, lower=True)
    V = rng.standard_normal(400) * 10.0 ** rng.integers(-30, 30, 400)
    out["symmetric_real"] = write(os.path.join(d, "symmetric_real.mtx"),
                                  "%%MatrixMarket matrix coordinate real symmetric", (50, 50, 400),
                                  [(str(i + 1), str(j + 1), "%.17e" % v) for i, j, v in zip(I, J, V)], blank=True)
    I, J = _entries(rng, 64, 64, 500)
    out["pattern_general"] = write(os.path.join(d, "pattern_general.mtx"),
                                   "%%MatrixMarket matrix coordinate pattern general", (64, 64, 500),
                                   [(str(i + 1), str(j + 1)) for i, j in zip(I, J)])
    I, J = _entries(rng, 40, 40, 200, lower=True)
    out["pattern_symmetric"] = write(os.path.join(d, "pattern_symmetric.mtx"),
                                     "%%MatrixMarket MATRIX Coordinate Pattern Symmetric", (40, 40, 200),
                                     [(str(i + 1), str(j + 1)) for i, j in zip(I, J)], eol="\r\n")
    I, J = _entries(rng, 33, 45, 250)
    K = rng.integers(-1000, 1000, 250)
    out["integer_general"] = write(os.path.join(d, "integer_general.mtx"),
                                   "%%MatrixMarket matrix coordinate integer general", (33, 45, 250),
                                   [(str(i + 1), str(j + 1), str(k)) for i, j, k in zip(I, J, K)],
                                   comments=("%", "% two comment lines"))
    out["empty_rows"] = write(os.path.join(d, "empty_rows.mtx"), "%%MatrixMarket matrix coordinate real general",
                              (10, 10, 2), [("3", "3", "1.5"), ("9", "1", "2.5")])
    out["no_entries"] = write(os.path.join(d, "no_entries.mtx"), "%%MatrixMarket matrix coordinate real general",
                              (5, 7, 0), [])
    # a stencil written column-major (rows scrambled for the stable sort)
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace3d_7pt(12)
    n = len(rp) - 1
    row_of = np.repeat(np.arange(n), np.diff(rp))
    order = np.lexsort((row_of, col))
    out["laplace3d_12_colmajor"] = write(os.path.join(d, "laplace3d_12_colmajor.mtx"),
                                         "%%MatrixMarket matrix coordinate real general", (n, n, len(col)),
                                         [(str(row_of[k] + 1), str(col[k] + 1), repr(float(val[k]))) for k in order])
    return out


def rejected(d):
    """{name: path} of files the reference refuses."""
    out = {}
    e = [("1", "1", "1.0")]
    for name, banner in (("complex", "%%MatrixMarket matrix coordinate complex general"),
                         ("array", "%%MatrixMarket matrix array real general"),
                         ("hermitian", "%%MatrixMarket matrix coordinate real hermitian"),
                         ("skew", "%%MatrixMarket matrix coordinate real skew-symmetric"),
                         ("no_banner", "% MatrixMarket matrix coordinate real general")):
        out[name] = write(os.path.join(d, name + ".mtx"), banner, (2, 2, 1), e)
    return out


def truncated(d):
    """A file with fewer entries than its size line announces.  The reference
    does not refuse it: mm_read_unsymmetric_sparse returns MM_PREMATURE_EOF
    (12, examples/mmio.hpp:84), which read_from_mtx's `< 0` test
    (examples/matrix_structs.hpp:117-119) lets through, and the missing entries
    are read from uninitialised memory.  The oracle and the platform refuse it."""
    return write(os.path.join(d, "premature_eof.mtx"), "%%MatrixMarket matrix coordinate real general", (3, 3, 4),
                 [("1", "1", "1"), ("2", "2", "2")])
