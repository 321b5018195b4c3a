"""Seeded synthetic CRS matrices of the benchmark configurations (numpy, host).

All generators return ``(row_ptr int32[n+1], col int32[nnz], val[nnz])`` in
natural lexicographic row order with ascending columns in every row, unless
stated otherwise.  The same arrays feed the CUDA platform and the CPU
reference, so every comparison is made on identical inputs.

* :func:`laplace3d_7pt`   -- 7-point 3D Laplacian, diagonal 6, off-diagonals -1
                             (64^3: the plain CRS SpMV case; 96^3: SpGEMM C = A*A).
* :func:`lognormal_random` -- 2^22 x 2^22 irregular matrix: row lengths
                             round(LogNormal(mu, sigma)) clipped to [1, 4096]
                             with mu = ln(mean) - sigma^2/2 (distribution mean 16),
                             columns uniform without repeats, sorted; values U[-1,1].
* :func:`stencil27`        -- 27-point 3D stencil, values U[0.5,1], diagonal 27.
* :func:`laplace2d_5pt`    -- 5-point 2D Laplacian, diagonal 4, off-diagonals -1.
* :func:`poisson2d_app`    -- the same operator in the row layout of the solver
                             applications (examples/applications/
                             applications_common.hpp:61-111): in-row order left,
                             bottom, diagonal, top, right (not sorted).
* :func:`lower_triangle`   -- D+L split of a CRS matrix (entries with col <= row),
                             as examples/examples_common.hpp:282-398 extract_D_L_U.
* :func:`random_symmetric_permutation` -- P A P^T for a seeded random P with the
                             reference's apply_mat_perm semantics
                             (src/utils/permutations.hpp:820-861: row r is old row
                             perm[r], columns mapped through inv_perm, in-row order kept).
"""
from __future__ import annotations

import numpy as np


def _finish(rows_len: np.ndarray, col: np.ndarray, val: np.ndarray):
    n = len(rows_len)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(rows_len, out=rp[1:])
    if rp[-1] >= 2 ** 31:
        raise ValueError("matrix too large for int32 indices")
    return rp.astype(np.int32), col.astype(np.int32, copy=False), val


def _stencil(dims, offsets, diag_value, off_value_fn, dtype):
    """Generic box stencil on a grid `dims` (slowest first), natural ordering."""
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    coords = np.indices(dims).reshape(len(dims), -1)  # [ndim, n]
    strides = np.array([int(np.prod(dims[i + 1:])) for i in range(len(dims))], dtype=np.int64)
    offsets = sorted(offsets, key=lambda o: int(np.dot(o, strides)))
    masks, cols = [], []
    for o in offsets:
        ok = np.ones(n, dtype=bool)
        for d, od in enumerate(o):
            c = coords[d] + od
            ok &= (c >= 0) & (c < dims[d])
        masks.append(ok)
        cols.append(np.arange(n, dtype=np.int64) + int(np.dot(o, strides)))
    M = np.stack(masks, axis=1)  # [n, n_off]
    C = np.stack(cols, axis=1)
    lens = M.sum(axis=1)
    col = C[M]
    is_diag = np.stack([np.full(n, all(v == 0 for v in o)) for o in offsets], axis=1)[M]
    val = np.empty(len(col), dtype=dtype)
    val[is_diag] = diag_value
    n_off = int((~is_diag).sum())
    val[~is_diag] = off_value_fn(n_off)
    return _finish(lens, col, val)


def laplace3d_7pt(nx: int, dtype=np.float64):
    offs = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    return _stencil((nx, nx, nx), offs, 6.0, lambda m: np.full(m, -1.0), dtype)


def laplace2d_5pt(nx: int, dtype=np.float64):
    offs = [(0, 0), (-1, 0), (1, 0), (0, -1), (0, 1)]
    return _stencil((nx, nx), offs, 4.0, lambda m: np.full(m, -1.0), dtype)


def poisson2d_app(nx: int, dtype=np.float64):
    """create2DPoissonMatrixCRS(nx): row i*nx + j holds, in this order, the
    entries of row-1 (j > 0), row-nx (i > 0), the diagonal 4, row+nx
    (i < nx-1) and row+1 (j < nx-1), off-diagonals -1."""
    nx = int(nx)
    r = np.arange(nx * nx, dtype=np.int64)
    i, j = r // nx, r % nx
    parts = [(j > 0, r - 1, -1.0), (i > 0, r - nx, -1.0), (np.ones_like(r, bool), r, 4.0),
             (i < nx - 1, r + nx, -1.0), (j < nx - 1, r + 1, -1.0)]
    M = np.stack([p[0] for p in parts], axis=1)
    Cc = np.stack([p[1] for p in parts], axis=1)
    V = np.stack([np.full(len(r), p[2]) for p in parts], axis=1)
    return _finish(M.sum(axis=1), Cc[M], V[M].astype(dtype))


def stencil27(nx: int, seed: int = 2, dtype=np.float64):
    rng = np.random.default_rng(seed)
    offs = [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)]
    return _stencil((nx, nx, nx), offs, 27.0, lambda m: rng.uniform(0.5, 1.0, m), dtype)


def lognormal_lengths(n: int, mean: float = 16.0, sigma: float = 1.0, seed: int = 1, lmax: int = 4096,
                      n_cols: int | None = None) -> np.ndarray:
    rng = np.random.default_rng(seed)
    mu = np.log(mean) - 0.5 * sigma * sigma
    lens = np.clip(np.rint(rng.lognormal(mu, sigma, n)), 1, lmax).astype(np.int64)
    return np.minimum(lens, n_cols or n)


def lognormal_random(n: int = 1 << 22, mean: float = 16.0, sigma: float = 1.0, seed: int = 1,
                     dtype=np.float64, lmax: int = 4096, n_cols: int | None = None):
    """Irregular matrix of the CRS/BCRS/SELL-C-sigma SpMV configuration
    (n_cols defaults to n; a row block of a wider matrix when larger)."""
    rng = np.random.default_rng(seed)
    nc = int(n_cols or n)
    mu = np.log(mean) - 0.5 * sigma * sigma
    lens = np.clip(np.rint(rng.lognormal(mu, sigma, n)), 1, lmax).astype(np.int64)
    lens = np.minimum(lens, nc)
    nnz = int(lens.sum())
    row = np.repeat(np.arange(n, dtype=np.int64), lens)
    col = rng.integers(0, nc, nnz, dtype=np.int64)
    key = row * nc + col
    key.sort()
    col = key - row * nc
    # repeated columns inside a row are rare (~E[len^2]/2 in total): redraw them
    dup = np.nonzero(col[1:] == col[:-1])[0] + 1
    dup = dup[row[dup] == row[dup - 1]]
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=rp[1:])
    for r in np.unique(row[dup]):
        s, e = rp[r], rp[r + 1]
        seen = set()
        out = []
        for c in col[s:e]:
            while int(c) in seen:
                c = rng.integers(0, nc)
            seen.add(int(c))
            out.append(int(c))
        col[s:e] = np.sort(np.array(out, dtype=np.int64))
    val = rng.uniform(-1.0, 1.0, nnz).astype(dtype)
    return _finish(lens, col, val)


def lower_triangle(row_ptr, col, val):
    """D+L part (col <= row) of a CRS matrix, in-row order kept."""
    n = len(row_ptr) - 1
    lens = np.diff(row_ptr).astype(np.int64)
    row = np.repeat(np.arange(n, dtype=np.int64), lens)
    keep = col.astype(np.int64) <= row
    new_lens = np.bincount(row[keep], minlength=n)
    return _finish(new_lens, col[keep], val[keep])


def apply_sym_perm(row_ptr, col, val, perm):
    """P A P^T: row r <- old row perm[r], columns through inv_perm, order kept."""
    n = len(row_ptr) - 1
    perm = np.asarray(perm, dtype=np.int64)
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n)
    lens = np.diff(row_ptr).astype(np.int64)[perm]
    starts = row_ptr[:-1].astype(np.int64)[perm]
    idx = np.repeat(starts - np.concatenate([[0], np.cumsum(lens)[:-1]]), lens) + np.arange(int(lens.sum()))
    return _finish(lens, inv[col[idx]], val[idx])


def random_symmetric_permutation(row_ptr, col, val, seed: int = 3):
    n = len(row_ptr) - 1
    perm = np.random.default_rng(seed).permutation(n)
    return apply_sym_perm(row_ptr, col, val, perm) + (perm.astype(np.int32),)


def uniform_vector(n: int, seed: int, dtype=np.float64, lo=-1.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, n).astype(dtype)


def crs_bytes(n_rows: int, nnz: int, n_cols: int, vbytes: int) -> int:
    """Algorithmic HBM bytes of one CRS SpMV: val+col per entry, row_ptr, x, y."""
    return (vbytes + 4) * nnz + 4 * (n_rows + 1) + vbytes * n_cols + vbytes * n_rows
