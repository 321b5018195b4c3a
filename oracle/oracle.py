"""Python front end of the CPU checkers (TEST INFRASTRUCTURE ONLY).

Two libraries sit behind this module:

* ``liboracle.so`` -- the plain-C restatement of the reference algorithms
  (``oracle/smax_oracle.c``); always available once ``make -C oracle oracle``
  (or ``__graft_entry__.build()``) has run.
* ``_ref/libsmax_ref.so`` -- the unmodified SmaxKernels reference compiled from
  its own sources through ``oracle/ref_shim.cpp``; present only where the
  reference checkout was available at build time.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module.  The product package never does.

All arrays are numpy; indices int32, values float64 or float32.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "liboracle.so")
REF_SO = os.path.join(_HERE, "_ref", "libsmax_ref.so")

_P = C.c_void_p
_I64 = C.c_int64
_U64 = C.c_uint64
_INT = C.c_int


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _sfx(dtype):
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def _vbits(dtype):
    return 32 if np.dtype(dtype) == np.float32 else 64


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# --------------------------------------------------------------------------
# The C restatement
# --------------------------------------------------------------------------
class Oracle:
    """ctypes view of liboracle.so (functions documented in smax_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run: make -C oracle oracle)")
        self.lib = C.CDLL(path)
        L = self.lib
        for s in ("f64", "f32"):
            getattr(L, f"orc_spmv_crs_{s}").argtypes = [_I64, _P, _P, _P, _P, _P]
            getattr(L, f"orc_spmv_scs_{s}").argtypes = [_I64, _I64, _P, _P, _P, _P, _P, _P]
            getattr(L, f"orc_spmv_bcrs_{s}").argtypes = [_I64] * 5 + [_P, _P, _P, _INT, _P, _P]
            getattr(L, f"orc_spmm_{s}").argtypes = [_INT, _I64, _P, _P, _P, _I64, _P, _P]
            getattr(L, f"orc_spgemm_numeric_{s}").argtypes = [_I64, _P, _P, _P, _P, _P, _P, _I64, _P, _P, _P]
            getattr(L, f"orc_peel_diag_{s}").argtypes = [_I64, _P, _P, _P, _P, _P]
            getattr(L, f"orc_peel_diag_{s}").restype = _INT
            getattr(L, f"orc_sptrsv_{s}").argtypes = [_INT, _I64, _P, _P, _P, _P, _P, _P]
            getattr(L, f"orc_sptrsv_lvl_{s}").argtypes = [_INT, _INT, _P, _P, _P, _P, _P, _P, _P]
            getattr(L, f"orc_sptrsm_{s}").argtypes = [_INT, _INT, _I64, _P, _P, _P, _P, _I64, _P, _P]
            getattr(L, f"orc_scs_fill_{s}").argtypes = [_I64, _I64, _P, _P, _P, _P, _P, _I64, _P, _P]
            getattr(L, f"orc_bcrs_fill_{s}").argtypes = [_I64] * 5 + [_INT, _P, _P, _P, _P, _P, _P]
            getattr(L, f"orc_apply_mat_perm_{s}").argtypes = [_I64, _P, _P, _P, _P, _P, _P, _P, _P]
            getattr(L, f"orc_apply_vec_perm_{s}").argtypes = [_I64, _P, _P, _P]
        L.orc_spgemm_row_counts.argtypes = [_I64, _P, _P, _I64, _P, _P, _P]
        L.orc_spgemm_fill_cols.argtypes = [_I64, _P, _P, _I64, _P, _P, _P, _P]
        L.orc_scs_layout.argtypes = [_I64, _P, _I64, _I64, _P, _P, _P, C.POINTER(_I64)]
        L.orc_scs_layout.restype = _INT
        L.orc_bcrs_pattern.argtypes = [_I64, _I64, _P, _P, _I64, _I64, _P, _P]
        L.orc_bcrs_pattern.restype = _INT
        L.orc_build_symmetric.argtypes = [_I64, _P, _P, _P, _P]
        L.orc_levels_rs.argtypes = [_I64, _P, _P, _P]
        L.orc_levels_rs.restype = _INT
        L.orc_perm_bfs.argtypes = [_I64, _P, _P, _P, _P]
        L.orc_perm_bfs.restype = _INT
        L.orc_generate_perm.argtypes = [_I64, _P, _P, _INT, _P, _P, _P]
        L.orc_generate_perm.restype = _INT

    # -- SpMV ---------------------------------------------------------------
    def spmv_crs(self, row_ptr, col, val, x):
        n = len(row_ptr) - 1
        y = np.zeros(n, dtype=val.dtype)
        getattr(self.lib, f"orc_spmv_crs_{_sfx(val.dtype)}")(
            n, _p(_i32(col)), _p(_i32(row_ptr)), _p(val), _p(np.ascontiguousarray(x, val.dtype)), _p(y))
        return y

    def spmv_scs(self, C_, chunk_ptr, chunk_lengths, col, val, x, n_rows_padded):
        y = np.zeros(n_rows_padded, dtype=val.dtype)
        getattr(self.lib, f"orc_spmv_scs_{_sfx(val.dtype)}")(
            C_, len(chunk_lengths), _p(_i32(chunk_ptr)), _p(_i32(chunk_lengths)), _p(_i32(col)),
            _p(val), _p(np.ascontiguousarray(x, val.dtype)), _p(y))
        return y

    def spmv_bcrs(self, n_brows, bh, bw, hpad, wpad, row_ptr, col, val, col_major, x):
        y = np.zeros(n_brows * hpad, dtype=val.dtype)
        getattr(self.lib, f"orc_spmv_bcrs_{_sfx(val.dtype)}")(
            n_brows, bh, bw, hpad, wpad, _p(_i32(col)), _p(_i32(row_ptr)), _p(val),
            int(bool(col_major)), _p(np.ascontiguousarray(x, val.dtype)), _p(y))
        return y

    # -- SpMM ---------------------------------------------------------------
    def spmm(self, row_ptr, col, val, X, k, row_major=True):
        n = len(row_ptr) - 1
        Y = np.zeros(n * k, dtype=val.dtype)
        getattr(self.lib, f"orc_spmm_{_sfx(val.dtype)}")(
            int(bool(row_major)), n, _p(_i32(col)), _p(_i32(row_ptr)), _p(val), k,
            _p(np.ascontiguousarray(X, val.dtype).ravel()), _p(Y))
        return Y

    # -- SpGEMM -------------------------------------------------------------
    def spgemm(self, a_row_ptr, a_col, a_val, b_row_ptr, b_col, b_val, b_n_cols):
        n = len(a_row_ptr) - 1
        a_row_ptr, a_col, b_row_ptr, b_col = map(_i32, (a_row_ptr, a_col, b_row_ptr, b_col))
        cnt = np.zeros(n, dtype=np.int32)
        self.lib.orc_spgemm_row_counts(n, _p(a_col), _p(a_row_ptr), b_n_cols, _p(b_col), _p(b_row_ptr), _p(cnt))
        c_row_ptr = np.zeros(n + 1, dtype=np.int32)
        np.cumsum(cnt, out=c_row_ptr[1:])
        c_col = np.zeros(int(c_row_ptr[-1]), dtype=np.int32)
        self.lib.orc_spgemm_fill_cols(n, _p(a_col), _p(a_row_ptr), b_n_cols, _p(b_col), _p(b_row_ptr),
                                      _p(c_row_ptr), _p(c_col))
        c_val = np.zeros(len(c_col), dtype=a_val.dtype)
        getattr(self.lib, f"orc_spgemm_numeric_{_sfx(a_val.dtype)}")(
            n, _p(a_col), _p(a_row_ptr), _p(a_val), _p(b_col), _p(b_row_ptr), _p(b_val),
            b_n_cols, _p(c_col), _p(c_row_ptr), _p(c_val))
        return c_row_ptr, c_col, c_val

    # -- triangular solves --------------------------------------------------
    def peel_diag(self, row_ptr, col, val):
        """Returns (col', val', D) with each diagonal moved to its row end."""
        col = _i32(col).copy()
        val = val.copy()
        n = len(row_ptr) - 1
        D = np.zeros(n, dtype=val.dtype)
        bad = _I64(-1)
        rc = getattr(self.lib, f"orc_peel_diag_{_sfx(val.dtype)}")(
            n, _p(col), _p(_i32(row_ptr)), _p(val), _p(D), C.cast(C.pointer(bad), C.c_void_p))
        if rc != 0:
            raise ValueError(f"peel_diag: error {rc} at row {bad.value}")
        return col, val, D

    def sptrsv(self, row_ptr, col, val, b, lower=True, levels=None):
        """Solves with the reference semantics: diagonal peeled first, then the
        plain sweep, or the level sweep when `levels` (lvl_ptr) is given."""
        pcol, pval, D = self.peel_diag(row_ptr, col, val)
        rp = _i32(row_ptr)
        x = np.zeros(len(rp) - 1, dtype=val.dtype)
        bb = np.ascontiguousarray(b, val.dtype)
        if levels is None:
            getattr(self.lib, f"orc_sptrsv_{_sfx(val.dtype)}")(
                int(bool(lower)), len(x), _p(pcol), _p(rp), _p(pval), _p(D), _p(x), _p(bb))
        else:
            lp = _i32(levels)
            getattr(self.lib, f"orc_sptrsv_lvl_{_sfx(val.dtype)}")(
                int(bool(lower)), len(lp) - 1, _p(lp), _p(pcol), _p(rp), _p(pval), _p(D), _p(x), _p(bb))
        return x

    # -- adjoints (no reference counterpart) ----------------------------------
    @staticmethod
    def transpose(row_ptr, col, val, n_cols):
        """CRS of A^T with each row in ascending row order of A (a stable
        counting sort of the entries by column)."""
        rp = _i32(row_ptr)
        col = _i32(col)
        n = len(rp) - 1
        rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
        order = np.argsort(col, kind="stable")
        t_rp = np.zeros(n_cols + 1, dtype=np.int32)
        np.cumsum(np.bincount(col, minlength=n_cols), out=t_rp[1:])
        return t_rp, rows[order].astype(np.int32), np.ascontiguousarray(val[order])

    def spmv_adjoint(self, row_ptr, col, val, x, g, n_cols=None):
        """y = A x, loss gradient g = dL/dy: returns (A^T g, dval) with
        dval[k] = g[row(k)] * x[col(k)], A^T formed on the host."""
        n = len(row_ptr) - 1
        n_cols = n if n_cols is None else n_cols
        t_rp, t_col, t_val = self.transpose(row_ptr, col, val, n_cols)
        dx = self.spmv_crs(t_rp, t_col, t_val, np.ascontiguousarray(g, val.dtype))
        rows = np.repeat(np.arange(n), np.diff(_i32(row_ptr)))
        dval = np.asarray(g, val.dtype)[rows] * np.asarray(x, val.dtype)[_i32(col)]
        return dx, dval

    def sptrsv_adjoint(self, row_ptr, col, val, x, g, lower=True):
        """L x = b, loss gradient g = dL/dx: returns (lambda, dval) with
        L^T lambda = g (an upper solve for lower L, through the reference
        semantics) and dval[k] = -lambda[row(k)] * x[col(k)]."""
        n = len(row_ptr) - 1
        t_rp, t_col, t_val = self.transpose(row_ptr, col, val, n)
        lam = self.sptrsv(t_rp, t_col, t_val, np.ascontiguousarray(g, val.dtype), lower=not lower)
        rows = np.repeat(np.arange(n), np.diff(_i32(row_ptr)))
        dval = -lam[rows] * np.asarray(x, val.dtype)[_i32(col)]
        return lam, dval

    def sptrsm(self, row_ptr, col, val, B, k, lower=True, row_major=True):
        pcol, pval, D = self.peel_diag(row_ptr, col, val)
        rp = _i32(row_ptr)
        n = len(rp) - 1
        X = np.zeros(n * k, dtype=val.dtype)
        BB = np.ascontiguousarray(B, val.dtype).ravel()
        getattr(self.lib, f"orc_sptrsm_{_sfx(val.dtype)}")(
            int(bool(row_major)), int(bool(lower)), n, _p(pcol), _p(rp), _p(pval), _p(D), k, _p(X), _p(BB))
        return X

    # -- conversions --------------------------------------------------------
    def scs(self, row_ptr, col, val, C_, sigma):
        """convert_crs_to_scs: returns dict with the reference's 13 SCS fields."""
        rp = _i32(row_ptr)
        n = len(rp) - 1
        n_chunks = (n + C_ - 1) // C_
        chunk_ptr = np.zeros(n_chunks + 1, dtype=np.int32)
        chunk_lengths = np.zeros(n_chunks, dtype=np.int32)
        perm = np.zeros(n, dtype=np.int32)
        ne = _I64(0)
        rc = self.lib.orc_scs_layout(n, _p(rp), C_, sigma, _p(chunk_ptr), _p(chunk_lengths), _p(perm),
                                     C.pointer(ne))
        if rc != 0:
            raise ValueError("scs layout")
        o_col = np.zeros(ne.value, dtype=np.int32)
        o_val = np.zeros(ne.value, dtype=val.dtype)
        getattr(self.lib, f"orc_scs_fill_{_sfx(val.dtype)}")(
            n, C_, _p(rp), _p(_i32(col)), _p(val), _p(chunk_ptr), _p(perm), ne.value, _p(o_col), _p(o_val))
        return dict(C=C_, sigma=sigma, n_rows=n, n_rows_padded=n_chunks * C_, n_chunks=n_chunks,
                    n_elements=ne.value, nnz=int(rp[-1]), chunk_ptr=chunk_ptr, chunk_lengths=chunk_lengths,
                    col=o_col, val=o_val, perm=perm)

    def bcrs(self, row_ptr, col, val, n_cols, bh, bw, hpad, wpad, col_major):
        rp = _i32(row_ptr)
        n = len(rp) - 1
        nb = n // bh
        brp = np.zeros(nb + 1, dtype=np.int32)
        rc = self.lib.orc_bcrs_pattern(n, n_cols, _p(rp), _p(_i32(col)), bh, bw, _p(brp), None)
        if rc != 0:
            raise ValueError("bcrs: block size does not divide the matrix")
        bcol = np.zeros(int(brp[-1]), dtype=np.int32)
        self.lib.orc_bcrs_pattern(n, n_cols, _p(rp), _p(_i32(col)), bh, bw, _p(brp), _p(bcol))
        bval = np.zeros(int(brp[-1]) * hpad * wpad, dtype=val.dtype)
        getattr(self.lib, f"orc_bcrs_fill_{_sfx(val.dtype)}")(
            nb, bh, bw, hpad, wpad, int(bool(col_major)), _p(rp), _p(_i32(col)), _p(val), _p(brp), _p(bcol),
            _p(bval))
        return dict(n_rows=nb, n_cols=n_cols // bw, n_blocks=int(brp[-1]), b_height=bh, b_width=bw,
                    height_pad=hpad, width_pad=wpad, row_ptr=brp, col=bcol, val=bval)

    # -- levels / permutations ----------------------------------------------
    def build_symmetric(self, row_ptr, col):
        rp = _i32(row_ptr)
        n = len(rp) - 1
        srp = np.zeros(n + 1, dtype=np.int32)
        self.lib.orc_build_symmetric(n, _p(rp), _p(_i32(col)), _p(srp), None)
        scol = np.zeros(int(srp[-1]), dtype=np.int32)
        self.lib.orc_build_symmetric(n, _p(rp), _p(_i32(col)), _p(srp), _p(scol))
        return srp, scol

    PERM_TYPES = {"BFS": 0, "RS": 1, "NONE": 2}

    def generate_perm(self, row_ptr, col, type_="RS"):
        """Returns (perm, inv_perm, lvl_ptr) as generate_perm leaves them."""
        rp = _i32(row_ptr)
        n = len(rp) - 1
        perm = np.zeros(n, dtype=np.int32)
        inv = np.zeros(n, dtype=np.int32)
        lvl_ptr = np.zeros(n + 2, dtype=np.int32)
        nl = self.lib.orc_generate_perm(n, _p(rp), _p(_i32(col)), self.PERM_TYPES[type_], _p(perm), _p(inv),
                                        _p(lvl_ptr))
        if nl < 0:
            raise ValueError("generate_perm")
        return perm, inv, lvl_ptr[: nl + 1].copy()

    # -- colourings (one OpenMP thread's results) ------------------------------
    @staticmethod
    def colour_sc(srp, scol):
        """generate_color_perm (src/utils/permutations.hpp:588-647) with one
        thread, on the symmetric pattern: (n_colours, colour[n])."""
        from collections import deque
        n = len(srp) - 1
        srp, scol = list(map(int, srp)), list(map(int, scol))
        color = [-2] * n
        usable = [-1] * n
        q = deque()
        for s_ in range(n):
            if all(scol[j] >= s_ for j in range(srp[s_], srp[s_ + 1])):
                q.append(s_)
                color[s_] = -1
        max_color = 0
        while q:
            u = q.popleft()
            for j in range(srp[u], srp[u + 1]):
                v = scol[j]
                if color[v] == -2:
                    color[v] = -1
                    q.append(v)
                elif color[v] >= 0:
                    usable[color[v]] = u
            for c in range(n):
                if usable[c] != u:
                    color[u] = c
                    max_color = max(max_color, c)
                    break
        return max_color + 1, np.array(color, dtype=np.int32)

    @staticmethod
    def colour_pc(srp, scol):
        """generate_color_perm_par (:649-714) with one thread: rows in order,
        each the smallest colour its neighbours do not hold (unset = -1)."""
        n = len(srp) - 1
        srp, scol = list(map(int, srp)), list(map(int, scol))
        colors = [-1] * n
        max_color = 0
        for row in range(n):
            forbidden = {colors[scol[j]] for j in range(srp[row], srp[row + 1])}
            spec = 0
            while spec in forbidden:
                spec += 1
            colors[row] = spec
            max_color = max(max_color, spec)
        return max_color + 1, np.array(colors, dtype=np.int32)

    @staticmethod
    def colour_balance(srp, scol, colors, num_colors):
        """generate_color_perm_bal (:716-792) with one thread, in place on a PC
        colouring.  The reference's search reads color_size past num_colors
        when every colour is ruled out; it then never moves the row, which is
        what stopping the search at num_colors gives."""
        n = len(srp) - 1
        srp, scol = list(map(int, srp)), list(map(int, scol))
        colors = [int(c) for c in colors]
        b = float(n // num_colors)
        size = [0] * num_colors
        for c in colors:
            size[c] += 1
        for row in range(n):
            if size[colors[row]] <= b:
                continue
            forbidden = {colors[scol[j]] for j in range(srp[row], srp[row + 1])}
            spec = 0
            while spec < num_colors and (spec in forbidden or size[spec] >= b):
                spec += 1
            if spec >= num_colors:
                continue
            size[colors[row]] -= 1
            colors[row] = spec
            size[spec] += 1
        return num_colors, np.array(colors, dtype=np.int32)

    @staticmethod
    def colours_valid(row_ptr, col, colors):
        """sanity_check_perm (:794-818)."""
        n = len(row_ptr) - 1
        for r in range(n):
            for j in range(int(row_ptr[r]), int(row_ptr[r + 1])):
                c = int(col[j])
                if c < r and colors[r] == colors[c] and colors[r] != 0:
                    return False
        return True

    def colour_perm(self, row_ptr, col, type_):
        """generate_perm for "SC", "PC", "PC_BAL": (perm, inv_perm, lvl_ptr,
        colour) -- the identity stably sorted by colour, one level per colour."""
        srp, scol = self.build_symmetric(row_ptr, col)
        if type_ == "SC":
            nc, colour = self.colour_sc(srp, scol)
        else:
            nc, colour = self.colour_pc(srp, scol)
            if type_ == "PC_BAL":
                nc, colour = self.colour_balance(srp, scol, colour, nc)
        n = len(colour)
        perm = np.argsort(colour, kind="stable").astype(np.int32)
        inv = np.zeros(n, dtype=np.int32)
        inv[perm] = np.arange(n, dtype=np.int32)
        lvl_ptr = np.zeros(nc + 1, dtype=np.int32)
        np.cumsum(np.bincount(colour, minlength=nc)[:nc], out=lvl_ptr[1:])
        return perm, inv, lvl_ptr, colour

    def apply_mat_perm(self, row_ptr, col, val, perm, inv_perm):
        rp = _i32(row_ptr)
        n = len(rp) - 1
        prp = np.zeros(n + 1, dtype=np.int32)
        pcol = np.zeros(len(col), dtype=np.int32)
        pval = np.zeros(len(col), dtype=val.dtype)
        getattr(self.lib, f"orc_apply_mat_perm_{_sfx(val.dtype)}")(
            n, _p(rp), _p(_i32(col)), _p(val), _p(prp), _p(pcol), _p(pval), _p(_i32(perm)), _p(_i32(inv_perm)))
        return prp, pcol, pval

    def apply_vec_perm(self, vec, perm):
        out = np.zeros(len(perm), dtype=vec.dtype)
        getattr(self.lib, f"orc_apply_vec_perm_{_sfx(vec.dtype)}")(len(perm), _p(vec), _p(out), _p(_i32(perm)))
        return out

    # -- Matrix Market ingestion (examples/matrix_structs.hpp) -----------------
    @staticmethod
    def read_mtx(path):
        """COOMatrix::read_from_mtx without fast_matrix_market
        (examples/matrix_structs.hpp:52-180, mmio.cpp:56-163, mmio.hpp:127-214)
        and convert_coo_to_crs (:338-387): banner checks, '%' comment lines,
        the size line, entries in file order (pattern values 0.01), symmetric
        mirrors right after each off-diagonal entry, a stable sort by row and
        the row pointer by counting.  Returns (n_rows, n_cols, nnz, row_ptr,
        col, val); raises ValueError where the reference reports an error."""
        with open(path, "r") as f:
            text = f.read()
        lines = text.split("\n")
        tok = lines[0].split()
        if len(tok) < 5 or not tok[0].startswith("%%MatrixMarket"):
            raise ValueError("banner")
        obj, fmt, data, sym = (t.lower() for t in tok[1:5])
        if obj != "matrix" or fmt != "coordinate" or data not in ("real", "integer", "pattern") or \
                sym not in ("general", "symmetric"):
            raise ValueError("unsupported")
        i = 1
        while True:
            if i >= len(lines):
                raise ValueError("premature end of file")
            ln = lines[i]
            i += 1
            if ln.startswith("%"):
                continue
            parts = ln.split()
            if len(parts) >= 3:
                M, N, nz = (int(p) for p in parts[:3])
                break
            if parts:
                raise ValueError("size line")
        rest = " ".join(lines[i:]).split()
        step = 2 if data == "pattern" else 3
        if len(rest) < step * nz:
            raise ValueError("premature end of file")
        I, J, V = [], [], []
        for e in range(nz):
            r, c = int(rest[step * e]) - 1, int(rest[step * e + 1]) - 1
            v = 0.01 if data == "pattern" else float(rest[step * e + 2])
            I.append(r)
            J.append(c)
            V.append(v)
            if sym == "symmetric" and r != c:
                I.append(c)
                J.append(r)
                V.append(v)
        I = np.array(I, dtype=np.int64)
        order = np.argsort(I, kind="stable")
        row_ptr = np.zeros(M + 1, dtype=np.int32)
        np.cumsum(np.bincount(I, minlength=M)[:M], out=row_ptr[1:])
        return (M, N, len(I), row_ptr, np.array(J, dtype=np.int32)[order], np.array(V, dtype=np.float64)[order])

    # -- the solver applications (examples/applications) --------------------
    @staticmethod
    def infty_norm(v):
        """infty_vec_norm (applications_common.hpp:122-133): the largest |v_i|
        found by `>` comparisons from 0, so NaNs never win."""
        a = np.abs(np.asarray(v, dtype=np.float64))
        a = a[a > 0.0]
        return float(a.max()) if len(a) else 0.0

    @staticmethod
    def jacobi_peel(row_ptr, col, val):
        """peel_diag_crs of the Jacobi application (jacobi/utils.hpp:7-36): the
        last diagonal entry of each row swapped into the row's last slot;
        returns (col', val', D).  A missing or |a_ii| < 1e-16 diagonal raises."""
        rp = np.asarray(row_ptr, dtype=np.int64)
        n = len(rp) - 1
        col = np.array(col, dtype=np.int32)
        val = np.array(val)
        row_of = np.repeat(np.arange(n), np.diff(rp))
        d = np.nonzero(col == row_of)[0]
        last = np.full(n, -1, dtype=np.int64)
        np.maximum.at(last, row_of[d], d)
        if n and (last < 0).any():
            raise ValueError(f"No diag! (row {int(np.argmax(last < 0))})")
        D = val[last].copy() if n else np.zeros(0, dtype=val.dtype)
        if n and (np.abs(D) < 1e-16).any():
            raise ValueError("Zero diag!")
        end = rp[1:] - 1
        for arr in (col, val):
            t = arr[last].copy()
            arr[last] = arr[end]
            arr[end] = t
        return col, val, D

    @staticmethod
    def split_d_l_u(row_ptr, col, val):
        """extract_D_L_U (examples/examples_common.hpp:283-398): D+L = entries
        with col <= row, U = the rest, each row in its own entry order."""
        rp = np.asarray(row_ptr, dtype=np.int64)
        n = len(rp) - 1
        row_of = np.repeat(np.arange(n), np.diff(rp))
        low = np.asarray(col) <= row_of
        out = []
        for m in (low, ~low):
            r = np.zeros(n + 1, dtype=np.int32)
            np.cumsum(np.bincount(row_of[m], minlength=n), out=r[1:])
            out.append((r, np.asarray(col, dtype=np.int32)[m].copy(), np.asarray(val)[m].copy()))
        return out[0], out[1]

    def jacobi_app(self, row_ptr, col, val, b, x_init, tol=1e-8, max_iters=1000, check_length=5):
        """The loop of examples/applications/jacobi/jacobi.cpp:14-58 on the
        matrix as given (the application permutes it first, :82-93):
          x_old = x_new = x_init; r = |b - A x_new|_inf
          while r > tol and n < max_iters:
              x_new = A x_old                                  ("x_new <- Ax_old")
              x_new = (b - (x_new - D x_old)) / D              (normalize_x)
              swap(x_old, x_new); n += 1                       (swap_operands)
              if n % check_length == 0: r = |b - A P|_inf      (P: the first x_new)
        with A's diagonal moved to each row end (peel_diag_crs).  Returns
        (latest iterate, n, r, residual history)."""
        pcol, pval, D = self.jacobi_peel(row_ptr, col, val)
        rp = _i32(row_ptr)
        b = np.asarray(b, dtype=pval.dtype)
        x_old = np.array(x_init, dtype=pval.dtype)
        x_new = x_old.copy()
        P = x_new  # the buffer "tmp <- Ax" was registered with

        def resid():
            return self.infty_norm(b - self.spmv_crs(rp, pcol, pval, P))

        norm = resid()
        hist = [norm]
        n = 0
        while norm > tol and n < max_iters:
            x_new[:] = self.spmv_crs(rp, pcol, pval, x_old)
            diag_contrib = D * x_old
            offdiag_sum = x_new - diag_contrib
            x_new[:] = (b - offdiag_sum) / D
            x_old, x_new = x_new, x_old
            n += 1
            if n % check_length == 0:
                norm = resid()
                hist.append(norm)
        return x_old.copy(), n, norm, np.array(hist)

    def gauss_seidel_app(self, row_ptr, col, val, b, x_init, tol=1e-8, max_iters=1000, check_length=5):
        """The loop of examples/applications/gauss_seidel/gauss_seidel.cpp:13-50:
          r = |b - A x|_inf
          while r > tol and n < max_iters:
              tmp = b - U x; x = (D+L)^-1 tmp (the reference's plain forward
              sweep, sptrsv_cpu_crs_impl.hpp:9-55); n += 1
              if n % check_length == 0: r = |b - A x|_inf
        Returns (x, n, r, residual history)."""
        (lrp, lcol, lval), (urp, ucol, uval) = self.split_d_l_u(row_ptr, col, val)
        rp = _i32(row_ptr)
        val = np.asarray(val)
        b = np.asarray(b, dtype=val.dtype)
        x = np.array(x_init, dtype=val.dtype)

        def resid():
            return self.infty_norm(b - self.spmv_crs(rp, col, val, x))

        norm = resid()
        hist = [norm]
        n = 0
        while norm > tol and n < max_iters:
            tmp = b - self.spmv_crs(urp, ucol, uval, x)
            x = self.sptrsv(lrp, lcol, lval, tmp)
            n += 1
            if n % check_length == 0:
                norm = resid()
                hist.append(norm)
        return x, n, norm, np.array(hist)


# --------------------------------------------------------------------------
# The reference itself (oracle/_ref), where it was built
# --------------------------------------------------------------------------
class Reference:
    """ctypes view of oracle/_ref/libsmax_ref.so (see oracle/ref_shim.cpp)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run: make -C oracle ref)")
        self.lib = C.CDLL(path)
        L = self.lib
        L.ref_last_error.restype = C.c_char_p
        L.ref_set_threads.argtypes = [_INT]
        L.ref_set_threads.restype = _INT
        L.ref_free_int.argtypes = [_P]
        L.ref_free_val.argtypes = [_INT, _P]
        L.ref_spmv_crs.argtypes = [_INT, _U64, _U64, _U64, _P, _P, _P, _P, _P]
        L.ref_time_spmv_crs.argtypes = [_INT, _U64, _U64, _U64, _P, _P, _P, _P, _P, _INT, _INT]
        L.ref_time_spmv_crs.restype = C.c_double
        L.ref_spmv_scs.argtypes = [_INT] + [_U64] * 8 + [_P] * 7
        L.ref_time_spmv_scs.argtypes = [_INT] + [_U64] * 8 + [_P] * 7 + [_INT, _INT]
        L.ref_time_spmv_scs.restype = C.c_double
        L.ref_spmv_bcrs.argtypes = [_INT] + [_U64] * 7 + [_P, _P, _P, _INT, _P, _P]
        L.ref_time_spmv_bcrs.argtypes = [_INT] + [_U64] * 7 + [_P, _P, _P, _INT, _P, _P, _INT, _INT]
        L.ref_time_spmv_bcrs.restype = C.c_double
        L.ref_spmm.argtypes = [_INT, _INT, _U64, _U64, _U64, _P, _P, _P, _U64, _P, _P]
        L.ref_time_spmm.argtypes = [_INT, _INT, _U64, _U64, _U64, _P, _P, _P, _U64, _P, _P, _INT, _INT]
        L.ref_time_spmm.restype = C.c_double
        L.ref_spgemm.argtypes = [_INT, _U64, _U64, _U64, _P, _P, _P, _U64, _U64, _U64, _P, _P, _P, _P,
                                 C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]
        L.ref_time_spgemm.argtypes = [_INT, _U64, _U64, _U64, _P, _P, _P, _INT]
        L.ref_time_spgemm.restype = C.c_double
        L.ref_sptrsv.argtypes = [_INT, _INT, _INT, _U64, _U64, _U64, _P, _P, _P, _P, _P, _INT, _P]
        L.ref_time_sptrsv.argtypes = [_INT, _INT, _INT, _U64, _U64, _U64, _P, _P, _P, _P, _P, _INT, _P,
                                      _INT, _INT]
        L.ref_time_sptrsv.restype = C.c_double
        L.ref_sptrsm.argtypes = [_INT, _INT, _INT, _U64, _U64, _U64, _P, _P, _P, _U64, _P, _P]
        L.ref_time_sptrsm.argtypes = [_INT, _INT, _U64, _U64, _U64, _P, _P, _P, _U64, _P, _P, _INT, _INT]
        L.ref_time_sptrsm.restype = C.c_double
        L.ref_convert_crs_to_scs.argtypes = [_INT, _U64, _U64, _U64, _P, _P, _P, _U64, _U64, _P] + \
            [C.POINTER(_P)] * 5
        L.ref_convert_crs_to_bcrs.argtypes = [_INT, _U64, _U64, _U64, _P, _P, _P, _U64, _U64, _U64, _U64,
                                              _INT, _P] + [C.POINTER(_P)] * 3
        L.ref_build_symmetric_crs.argtypes = [_U64, _P, _P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_U64)]
        L.ref_generate_perm.argtypes = [_INT, _P, _P, _P, _P, C.c_char_p, C.POINTER(_INT), C.POINTER(_P)]
        L.ref_time_generate_perm.argtypes = [_INT, _P, _P, _P, _P, C.c_char_p]
        L.ref_time_generate_perm.restype = C.c_double
        L.ref_apply_mat_perm.argtypes = [_INT, _INT, _P, _P, _P, _P, _P, _P, _P, _P]
        L.ref_apply_vec_perm.argtypes = [_INT, _INT, _P, _P, _P]
        L.ref_read_mtx.argtypes = [C.c_char_p, C.POINTER(_U64), C.POINTER(_U64), C.POINTER(_U64),
                                   C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]
        for name in ("ref_jacobi", "ref_gauss_seidel"):
            f = getattr(L, name)
            f.argtypes = [_U64, _U64, _P, _P, _P, _P, _P, C.c_double, _INT, _INT, C.POINTER(_INT),
                          C.POINTER(C.c_double), _P, _INT, C.POINTER(_INT)]
            f.restype = C.c_double

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(f"reference error: {self.lib.ref_last_error().decode()}")

    def _app(self, fn, row_ptr, col, val, b, x_init, tol, max_iters, check_length):
        rp, col = _i32(row_ptr), _i32(col)
        val = np.ascontiguousarray(val, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.array(x_init, dtype=np.float64)
        cap = max_iters // max(check_length, 1) + 1
        hist = np.zeros(cap, dtype=np.float64)
        it, norm, nch = _INT(0), C.c_double(0.0), _INT(0)
        t = fn(len(rp) - 1, len(col), _p(col), _p(rp), _p(val), _p(b), _p(x), float(tol), int(max_iters),
               int(check_length), C.byref(it), C.byref(norm), _p(hist), cap, C.byref(nch))
        if t < 0:
            self._check(-1)
        return x, it.value, norm.value, hist[: min(nch.value, cap)], t

    def read_mtx(self, path):
        """The examples' reader + convert_coo_to_crs (ref_read_mtx):
        (n_rows, n_cols, nnz, row_ptr, col, val)."""
        nr, nc, nz = _U64(0), _U64(0), _U64(0)
        rp, col, val = _P(), _P(), _P()
        self._check(self.lib.ref_read_mtx(os.fsencode(path), C.byref(nr), C.byref(nc), C.byref(nz), C.byref(rp),
                                          C.byref(col), C.byref(val)))
        n, z = nr.value, nz.value
        return (n, nc.value, z, self._take_int(rp.value, n + 1), self._take_int(col.value, z),
                self._take_val(val.value, z, np.float64))

    def jacobi_app(self, row_ptr, col, val, b, x_init, tol=1e-8, max_iters=1000, check_length=5):
        """The Jacobi program's loop through the reference's kernels (ref_jacobi):
        (x, n_iters, residual, history, seconds in the loop)."""
        return self._app(self.lib.ref_jacobi, row_ptr, col, val, b, x_init, tol, max_iters, check_length)

    def gauss_seidel_app(self, row_ptr, col, val, b, x_init, tol=1e-8, max_iters=1000, check_length=5):
        """The Gauss-Seidel program's loop through the reference's kernels."""
        return self._app(self.lib.ref_gauss_seidel, row_ptr, col, val, b, x_init, tol, max_iters, check_length)

    def set_threads(self, n: int) -> int:
        return self.lib.ref_set_threads(n)

    def _take_int(self, p, n):
        a = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_int32)), shape=(n,)).copy() if n else \
            np.zeros(0, np.int32)
        self.lib.ref_free_int(p)
        return a

    def _take_val(self, p, n, dtype):
        ct = C.c_float if np.dtype(dtype) == np.float32 else C.c_double
        a = np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(n,)).copy() if n else np.zeros(0, dtype)
        self.lib.ref_free_val(_vbits(dtype), p)
        return a

    def spmv_crs(self, row_ptr, col, val, x, n_cols=None):
        rp, cl = _i32(row_ptr), _i32(col)
        n = len(rp) - 1
        y = np.zeros(n, dtype=val.dtype)
        x = np.ascontiguousarray(x, val.dtype)
        self._check(self.lib.ref_spmv_crs(_vbits(val.dtype), n, n_cols or len(x), len(cl), _p(cl), _p(rp),
                                          _p(val), _p(x), _p(y)))
        return y

    def time_spmv_crs(self, row_ptr, col, val, x, warm=3, reps=20):
        rp, cl = _i32(row_ptr), _i32(col)
        n = len(rp) - 1
        y = np.zeros(n, dtype=val.dtype)
        x = np.ascontiguousarray(x, val.dtype)
        t = self.lib.ref_time_spmv_crs(_vbits(val.dtype), n, len(x), len(cl), _p(cl), _p(rp), _p(val), _p(x),
                                       _p(y), warm, reps)
        if t < 0:
            self._check(-1)
        return t, y

    def spmv_scs(self, s, x):
        vs = max(s["n_rows_padded"], len(x))
        xx = np.zeros(vs, dtype=s["val"].dtype)
        xx[: len(x)] = x
        y = np.zeros(vs, dtype=s["val"].dtype)
        self._check(self.lib.ref_spmv_scs(
            _vbits(s["val"].dtype), s["C"], s["sigma"], s["n_rows"], s["n_rows_padded"], len(x), s["n_chunks"],
            s["n_elements"], s["nnz"], _p(_i32(s["chunk_ptr"])), _p(_i32(s["chunk_lengths"])),
            _p(_i32(s["col"])), _p(s["val"]), _p(_i32(s["perm"])), _p(xx), _p(y)))
        return y

    def spmv_bcrs(self, b, x, col_major):
        y = np.zeros(b["n_rows"] * b["height_pad"], dtype=b["val"].dtype)
        x = np.ascontiguousarray(x, b["val"].dtype)
        self._check(self.lib.ref_spmv_bcrs(
            _vbits(b["val"].dtype), b["n_rows"], b["n_cols"], b["n_blocks"], b["b_height"], b["b_width"],
            b["height_pad"], b["width_pad"], _p(_i32(b["col"])), _p(_i32(b["row_ptr"])), _p(b["val"]),
            int(bool(col_major)), _p(x), _p(y)))
        return y

    def spmm(self, row_ptr, col, val, X, k, row_major=True, n_cols=None):
        rp, cl = _i32(row_ptr), _i32(col)
        n = len(rp) - 1
        Y = np.zeros(n * k, dtype=val.dtype)
        X = np.ascontiguousarray(X, val.dtype).ravel()
        self._check(self.lib.ref_spmm(_vbits(val.dtype), int(bool(row_major)), n, n_cols or n, len(cl), _p(cl),
                                      _p(rp), _p(val), k, _p(X), _p(Y)))
        return Y

    def spgemm(self, a_row_ptr, a_col, a_val, b_row_ptr, b_col, b_val, a_n_cols, b_n_cols):
        arp, acl, brp, bcl = map(_i32, (a_row_ptr, a_col, b_row_ptr, b_col))
        meta = np.zeros(3, dtype=np.uint64)
        pc, pr, pv = _P(), _P(), _P()
        self._check(self.lib.ref_spgemm(_vbits(a_val.dtype), len(arp) - 1, a_n_cols, len(acl), _p(acl), _p(arp),
                                        _p(a_val), len(brp) - 1, b_n_cols, len(bcl), _p(bcl), _p(brp), _p(b_val),
                                        _p(meta), C.byref(pc), C.byref(pr), C.byref(pv)))
        nr, nc, nz = (int(v) for v in meta)
        return (self._take_int(pr.value, nr + 1), self._take_int(pc.value, nz),
                self._take_val(pv.value, nz, a_val.dtype), nr, nc)

    def sptrsv(self, row_ptr, col, val, b, upper=False, levels=None):
        """Runs the reference SpTRSV on COPIES of col/val (it mutates them)."""
        rp = _i32(row_ptr)
        cl = _i32(col).copy()
        vv = val.copy()
        n = len(rp) - 1
        x = np.zeros(n, dtype=val.dtype)
        bb = np.ascontiguousarray(b, val.dtype).copy()
        lp = _i32(levels) if levels is not None else np.zeros(1, np.int32)
        self._check(self.lib.ref_sptrsv(_vbits(val.dtype), int(bool(upper)), int(levels is not None), n, n,
                                        len(cl), _p(cl), _p(rp), _p(vv), _p(x), _p(bb), len(lp) - 1, _p(lp)))
        return x

    def time_sptrsv(self, row_ptr, col, val, b, upper=False, levels=None, warm=2, reps=10):
        rp = _i32(row_ptr)
        cl = _i32(col).copy()
        vv = val.copy()
        n = len(rp) - 1
        x = np.zeros(n, dtype=val.dtype)
        bb = np.ascontiguousarray(b, val.dtype).copy()
        lp = _i32(levels) if levels is not None else np.zeros(1, np.int32)
        t = self.lib.ref_time_sptrsv(_vbits(val.dtype), int(bool(upper)), int(levels is not None), n, n, len(cl),
                                     _p(cl), _p(rp), _p(vv), _p(x), _p(bb), len(lp) - 1, _p(lp), warm, reps)
        if t < 0:
            self._check(-1)
        return t, x

    # -- timers (seconds per apply after `warm` applies) -----------------------
    def _t(self, t):
        if t < 0:
            self._check(-1)
        return t

    def time_spmv_scs(self, s, x, warm=1, reps=10):
        vs = max(s["n_rows_padded"], len(x))
        xx = np.zeros(vs, dtype=s["val"].dtype)
        xx[: len(x)] = x
        y = np.zeros(vs, dtype=s["val"].dtype)
        return self._t(self.lib.ref_time_spmv_scs(
            _vbits(s["val"].dtype), s["C"], s["sigma"], s["n_rows"], s["n_rows_padded"], len(x), s["n_chunks"],
            s["n_elements"], s["nnz"], _p(_i32(s["chunk_ptr"])), _p(_i32(s["chunk_lengths"])),
            _p(_i32(s["col"])), _p(s["val"]), _p(_i32(s["perm"])), _p(xx), _p(y), warm, reps))

    def time_spmv_bcrs(self, b, x, col_major=False, warm=1, reps=10):
        y = np.zeros(b["n_rows"] * b["height_pad"], dtype=b["val"].dtype)
        x = np.ascontiguousarray(x, b["val"].dtype)
        return self._t(self.lib.ref_time_spmv_bcrs(
            _vbits(b["val"].dtype), b["n_rows"], b["n_cols"], b["n_blocks"], b["b_height"], b["b_width"],
            b["height_pad"], b["width_pad"], _p(_i32(b["col"])), _p(_i32(b["row_ptr"])), _p(b["val"]),
            int(bool(col_major)), _p(x), _p(y), warm, reps))

    def time_spmm(self, row_ptr, col, val, X, k, row_major=True, warm=1, reps=10):
        rp, cl = _i32(row_ptr), _i32(col)
        n = len(rp) - 1
        Y = np.zeros(n * k, dtype=val.dtype)
        X = np.ascontiguousarray(X, val.dtype).ravel()
        return self._t(self.lib.ref_time_spmm(_vbits(val.dtype), int(bool(row_major)), n, n, len(cl), _p(cl),
                                              _p(rp), _p(val), k, _p(X), _p(Y), warm, reps))

    def time_spgemm(self, row_ptr, col, val, reps=3):
        """C = A*A: seconds of apply() (symbolic + numeric phases)."""
        rp, cl = _i32(row_ptr), _i32(col)
        n = len(rp) - 1
        return self._t(self.lib.ref_time_spgemm(_vbits(val.dtype), n, n, len(cl), _p(cl), _p(rp), _p(val), reps))

    def time_sptrsm(self, row_ptr, col, val, B, k, row_major=True, warm=1, reps=5):
        rp = _i32(row_ptr)
        cl = _i32(col).copy()
        vv = val.copy()
        n = len(rp) - 1
        X = np.zeros(n * k, dtype=val.dtype)
        BB = np.ascontiguousarray(B, val.dtype).ravel().copy()
        return self._t(self.lib.ref_time_sptrsm(_vbits(val.dtype), int(bool(row_major)), n, n, len(cl), _p(cl),
                                                _p(rp), _p(vv), k, _p(X), _p(BB), warm, reps))

    def sptrsm(self, row_ptr, col, val, B, k, row_major=True):
        rp = _i32(row_ptr)
        cl = _i32(col).copy()
        vv = val.copy()
        n = len(rp) - 1
        X = np.zeros(n * k, dtype=val.dtype)
        BB = np.ascontiguousarray(B, val.dtype).ravel().copy()
        self._check(self.lib.ref_sptrsm(_vbits(val.dtype), int(bool(row_major)), 0, n, n, len(cl), _p(cl), _p(rp),
                                        _p(vv), k, _p(X), _p(BB)))
        return X

    def scs(self, row_ptr, col, val, C_, sigma, n_cols=None):
        rp, cl = _i32(row_ptr), _i32(col)
        n = len(rp) - 1
        meta = np.zeros(6, dtype=np.uint64)
        ptrs = [_P() for _ in range(5)]
        self._check(self.lib.ref_convert_crs_to_scs(_vbits(val.dtype), n, n_cols or n, len(cl), _p(cl), _p(rp),
                                                    _p(val), C_, sigma, _p(meta), *[C.byref(p) for p in ptrs]))
        nr, npad, nc, nch, ne, nz = (int(v) for v in meta)
        return dict(C=C_, sigma=sigma, n_rows=nr, n_rows_padded=npad, n_cols=nc, n_chunks=nch, n_elements=ne,
                    nnz=nz, chunk_ptr=self._take_int(ptrs[0].value, nch + 1),
                    chunk_lengths=self._take_int(ptrs[1].value, nch), col=self._take_int(ptrs[2].value, ne),
                    val=self._take_val(ptrs[3].value, ne, val.dtype), perm=self._take_int(ptrs[4].value, nr))

    def bcrs(self, row_ptr, col, val, n_cols, bh, bw, hpad, wpad, col_major):
        rp, cl = _i32(row_ptr), _i32(col)
        n = len(rp) - 1
        meta = np.zeros(7, dtype=np.uint64)
        ptrs = [_P() for _ in range(3)]
        self._check(self.lib.ref_convert_crs_to_bcrs(_vbits(val.dtype), n, n_cols, len(cl), _p(cl), _p(rp), _p(val),
                                                     bh, bw, hpad, wpad, int(bool(col_major)), _p(meta),
                                                     *[C.byref(p) for p in ptrs]))
        nr, nc, nb, bh_, bw_, hp, wp = (int(v) for v in meta)
        return dict(n_rows=nr, n_cols=nc, n_blocks=nb, b_height=bh_, b_width=bw_, height_pad=hp, width_pad=wp,
                    col=self._take_int(ptrs[0].value, nb), row_ptr=self._take_int(ptrs[1].value, nr + 1),
                    val=self._take_val(ptrs[2].value, nb * hp * wp, val.dtype))

    def build_symmetric(self, row_ptr, col):
        rp, cl = _i32(row_ptr), _i32(col)
        n = len(rp) - 1
        pr, pc, nz = _P(), _P(), _U64(0)
        self._check(self.lib.ref_build_symmetric_crs(n, _p(rp), _p(cl), C.byref(pr), C.byref(pc), C.byref(nz)))
        return self._take_int(pr.value, n + 1), self._take_int(pc.value, nz.value)

    def generate_perm(self, row_ptr, col, type_="RS"):
        rp, cl = _i32(row_ptr), _i32(col)
        n = len(rp) - 1
        perm = np.zeros(n, dtype=np.int32)
        inv = np.zeros(n, dtype=np.int32)
        nl = _INT(0)
        plp = _P()
        self._check(self.lib.ref_generate_perm(n, _p(rp), _p(cl), _p(perm), _p(inv), type_.encode(), C.byref(nl),
                                               C.byref(plp)))
        return perm, inv, self._take_int(plp.value, nl.value + 1)

    def apply_mat_perm(self, row_ptr, col, val, perm, inv_perm):
        rp, cl = _i32(row_ptr), _i32(col)
        n = len(rp) - 1
        prp = np.zeros(n + 1, dtype=np.int32)
        pcol = np.zeros(len(cl), dtype=np.int32)
        pval = np.zeros(len(cl), dtype=val.dtype)
        self._check(self.lib.ref_apply_mat_perm(_vbits(val.dtype), n, _p(rp), _p(cl), _p(val), _p(prp), _p(pcol),
                                                _p(pval), _p(_i32(perm)), _p(_i32(inv_perm))))
        return prp, pcol, pval


def oracle_available() -> bool:
    return os.path.exists(ORACLE_SO)


def reference_available() -> bool:
    return os.path.exists(REF_SO)
