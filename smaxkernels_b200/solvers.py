"""Device-resident Jacobi and Gauss-Seidel: the reference's solver applications.

The reference ships two iterative solvers as example programs
(examples/applications/jacobi/jacobi.cpp:14-130 and
gauss_seidel/gauss_seidel.cpp:13-111) that call ``run()`` on SpMV / SpTRSV
kernels once per iteration and do the vector arithmetic on the host.  Here
the same loop runs on the GPU through the C ABI's ``smax_solver_*`` (the loop,
the residual rule and the buffer swap of Jacobi are documented in
include/smax_b200.h):

    s = Solver("jacobi", row_ptr, col, val)
    stats = s.solve(b, x)             # x: initial guess in, solution out
    s.history()                       # residuals at every check

Arrays are numpy arrays or torch tensors, on the host or on the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib
from .interface import _ptr

KINDS = {"jacobi": 0, "gauss_seidel": 1}
MODES = {"device_loop": 0, "graph_blocks": 1, "plain": 2}


def _dtype_of(a):
    if hasattr(a, "dtype") and not isinstance(a, np.ndarray):
        import torch
        return np.float64 if a.dtype == torch.float64 else (np.float32 if a.dtype == torch.float32 else None)
    return a.dtype.type if a.dtype in (np.float64, np.float32) else None


class Solver:
    """One solver on one square CRS matrix (int32 indices)."""

    def __init__(self, kind: str, row_ptr, col, val, n_rows: int | None = None):
        if kind not in KINDS:
            raise ValueError(f"kind must be one of {sorted(KINDS)}")
        self.kind = kind
        if isinstance(row_ptr, np.ndarray):
            row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
            col = np.ascontiguousarray(col, dtype=np.int32)
            val = np.ascontiguousarray(val)
        vt = _dtype_of(val)
        if vt is None:
            raise TypeError("values must be float64 or float32")
        self.dtype = vt
        n = int(n_rows) if n_rows is not None else len(row_ptr) - 1
        nnz = int(len(col))
        self.n_rows = n
        ft = 1 if vt == np.float64 else 0
        self._h = C.c_void_p()
        check(lib.smax_solver_create(C.byref(self._h), KINDS[kind], ft, n, nnz, _ptr(row_ptr), _ptr(col),
                                     _ptr(val)))

    def solve(self, b, x, tol: float = 1e-8, max_iters: int = 1000, check_length: int = 5,
              mode: str = "device_loop", stream: int | None = None) -> dict:
        """Runs the application's loop from the initial guess in x and leaves
        the solution in x; returns smax_solver_stats as a dict."""
        for a in (b, x):
            if _dtype_of(a) != self.dtype:
                raise TypeError("b and x must have the solver's value type")
            if len(a) < self.n_rows:
                raise ValueError("b and x need n_rows values")
        opts = _lib.SolverOpts(float(tol), int(max_iters), int(check_length), MODES[mode])
        stats = _lib.SolverStats()
        check(lib.smax_solver_solve(self._h, _ptr(b), _ptr(x), C.byref(opts), C.byref(stats),
                                    C.c_void_p(stream) if stream else None))
        return _lib.struct_dict(stats)

    def history(self) -> np.ndarray:
        """The residuals of the last solve, in the order they were measured."""
        count = C.c_int(0)
        check(lib.smax_solver_get_history(self._h, None, 0, C.byref(count)))
        out = np.zeros(min(count.value, 1 << 20), dtype=np.float64)  # the first 2^20 are kept
        if len(out):
            check(lib.smax_solver_get_history(self._h, out.ctypes.data_as(C.c_void_p), len(out),
                                              C.byref(count)))
        return out

    def close(self):
        if self._h:
            lib.smax_solver_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def jacobi(row_ptr, col, val, b, x, **kw) -> dict:
    with Solver("jacobi", row_ptr, col, val) as s:
        return s.solve(b, x, **kw)


def gauss_seidel(row_ptr, col, val, b, x, **kw) -> dict:
    with Solver("gauss_seidel", row_ptr, col, val) as s:
        return s.solve(b, x, **kw)
