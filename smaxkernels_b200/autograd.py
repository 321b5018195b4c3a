"""torch.autograd over the platform's CRS SpMV and SpTRSV kernels.

The reference has no derivatives; this module adds them on top of the C ABI's
reverse-mode entry (``smax_kernel_adjoint``):

* ``spmv(A, val, x)``   -> y = A(val) x;   grads: dval[k] = g[row k] x[col k],
  dx = A^T g (a warp-stream SpMV with the transposed copy).
* ``sptrsv(L, val, b)`` -> x = L(val)^-1 b; grads: db = lambda with
  L^T lambda = g (the forward level sets swept in reverse),
  dval[k] = -lambda[row k] x[col k].

A :class:`SparsePattern` owns one kernel object with the pattern resident in
HBM; values are differentiable tensors that are copied into the device copy
(``smax_kernel_update_A_values``) on every call.  Every call runs on
torch's current stream, and the kernel object's operand buffers stay fixed so
the solves' CUDA graphs are captured once.

``val`` is in the caller's entry order.  For triangular solves the device copy
keeps each diagonal last in its row (the reference's peel,
src/kernels/sptrsv/sptrsv_cpu/sptrsv_cpu_crs_helpers_impl.hpp:9-38); the
pattern object holds that permutation and applies it both ways.
"""
from __future__ import annotations

import numpy as np
import torch

from .interface import FloatType, Interface, IntType, KernelType, PlatformType


def _peel_order(row_ptr: np.ndarray, col: np.ndarray) -> np.ndarray:
    """Entry permutation that swaps each row's last diagonal entry with the
    row's last entry (identity where the diagonal is already last)."""
    n = len(row_ptr) - 1
    lens = np.diff(row_ptr)
    if n and (lens <= 0).any():
        raise ValueError(f"row {int(np.argmax(lens <= 0))} has no entries (no diagonal)")
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    idx = np.arange(len(col), dtype=np.int64)
    cand = np.where(col == rows, idx, -1)
    last = np.maximum.reduceat(cand, row_ptr[:-1].astype(np.int64)) if n else np.zeros(0, np.int64)
    if (last < 0).any():
        raise ValueError(f"row {int(np.argmax(last < 0))} has no diagonal entry")
    end = row_ptr[1:].astype(np.int64) - 1
    perm = idx.copy()
    perm[last] = end
    perm[end] = last
    return perm


class SparsePattern:
    """A CRS pattern on the GPU, for differentiable SpMV ("spmv") or
    triangular solves ("sptrsv", lower unless upper=True)."""

    def __init__(self, row_ptr, col, n_cols=None, *, kind: str = "spmv", upper: bool = False,
                 dtype: torch.dtype = torch.float64, device="cuda"):
        if kind not in ("spmv", "sptrsv"):
            raise ValueError("kind must be 'spmv' or 'sptrsv'")
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        col = np.ascontiguousarray(col, dtype=np.int32)
        self.n_rows = len(self.row_ptr) - 1
        self.n_cols = self.n_rows if n_cols is None else int(n_cols)
        self.nnz = len(col)
        self.kind = kind
        self.dtype = dtype
        self.device = torch.device(device)
        if kind == "sptrsv" and self.n_cols != self.n_rows:
            raise ValueError("triangular solves need a square pattern")
        if kind == "sptrsv":
            order = _peel_order(self.row_ptr, col)
            self._order = torch.from_numpy(order).to(self.device)
            self.col = np.ascontiguousarray(col[order])
        else:
            self._order = None
            self.col = col
        ft = FloatType.FLOAT64 if dtype == torch.float64 else FloatType.FLOAT32
        kt = KernelType.SPMV if kind == "spmv" else KernelType.SPTRSV
        self._iface = Interface()
        self._iface.register_kernel("op", kt, PlatformType.CUDA, IntType.INT32, ft)
        self.k = self._iface.kernel("op")
        if upper:
            self.k.set_mat_upper_triang(True)
        npdt = np.float64 if dtype == torch.float64 else np.float32
        # placeholder values (unit diagonal for solves) until the first call
        self._val_init = np.ones(self.nnz, dtype=npdt)
        opts = dict(dtype=dtype, device=self.device)
        if kind == "spmv":
            self._in = torch.zeros(self.n_cols, **opts)    # B: x
            self._out = torch.zeros(self.n_rows, **opts)   # C: y
            self.k.register_A(self.n_rows, self.n_cols, self.nnz, self.col, self.row_ptr, self._val_init)
            self.k.register_B(self.n_cols, self._in)
            self.k.register_C(self.n_rows, self._out)
        else:
            self._in = torch.zeros(self.n_rows, **opts)    # C: b
            self._out = torch.zeros(self.n_rows, **opts)   # B: x
            self.k.register_A(self.n_rows, self.n_cols, self.nnz, self.col, self.row_ptr, self._val_init)
            self.k.register_B(self.n_rows, self._out)
            self.k.register_C(self.n_rows, self._in)
        self._g = torch.zeros(self.n_rows, **opts)
        self._din = torch.zeros(self.n_cols, **opts)
        self._dval = torch.zeros(self.nnz, **opts)
        self._bind_stream()
        self.k.initialize()

    # -- plumbing ---------------------------------------------------------
    def _bind_stream(self):
        self.k.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def _set_values(self, val: torch.Tensor):
        if val.shape != (self.nnz,):
            raise ValueError(f"expected {self.nnz} values, got shape {tuple(val.shape)}")
        # copied on every call (an nnz-sized device copy): edits through
        # .data leave no trace a cache could check
        v = val.detach().to(device=self.device, dtype=self.dtype)
        v = (v[self._order] if self._order is not None else v).contiguous()
        self.k.update_A_values(v)
        self._keep = v  # the copy is asynchronous on the stream: keep the source alive

    def _to_user_order(self, dval_dev: torch.Tensor) -> torch.Tensor:
        if self._order is None:
            return dval_dev.clone()
        out = torch.empty_like(dval_dev)
        out[self._order] = dval_dev
        return out

    # -- forward passes (no autograd) ----------------------------------------
    def forward(self, val: torch.Tensor, inp: torch.Tensor) -> torch.Tensor:
        self._bind_stream()
        self._set_values(val)
        self._in.copy_(inp.detach().reshape(-1))
        self.k.apply()
        return self._out.clone()

    def backward(self, val: torch.Tensor, x: torch.Tensor, g: torch.Tensor, need_val: bool, need_in: bool):
        """(dval in the caller's entry order or None, d_in or None)."""
        self._bind_stream()
        self._set_values(val)
        self._g.copy_(g.reshape(-1))
        xs = x.detach().to(self.dtype).contiguous()
        need_din = need_in or self.kind == "sptrsv"  # the solve's dval needs lambda
        self.k.adjoint(self._g, self._din if need_din else None, self._dval if need_val else None, x=xs)
        dval = self._to_user_order(self._dval) if need_val else None
        din = self._din.clone() if need_in else None
        return dval, din


class _SpMV(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A: SparsePattern, val, x):
        y = A.forward(val, x)
        ctx.A = A
        ctx.save_for_backward(val, x)
        return y

    @staticmethod
    def backward(ctx, gy):
        val, x = ctx.saved_tensors
        dval, dx = ctx.A.backward(val, x, gy.contiguous(), ctx.needs_input_grad[1], ctx.needs_input_grad[2])
        return None, dval, dx


class _SpTRSV(torch.autograd.Function):
    @staticmethod
    def forward(ctx, L: SparsePattern, val, b):
        x = L.forward(val, b)
        ctx.L = L
        ctx.save_for_backward(val, x)
        return x

    @staticmethod
    def backward(ctx, gx):
        val, x = ctx.saved_tensors
        dval, db = ctx.L.backward(val, x, gx.contiguous(), ctx.needs_input_grad[1], ctx.needs_input_grad[2])
        return None, dval, db


def spmv(A: SparsePattern, val: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
    """y = A(val) x, differentiable in val and x."""
    if A.kind != "spmv":
        raise ValueError("pattern was not created for spmv")
    return _SpMV.apply(A, val, x)


def sptrsv(L: SparsePattern, val: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """x = L(val)^-1 b, differentiable in val and b."""
    if L.kind != "sptrsv":
        raise ValueError("pattern was not created for sptrsv")
    return _SpTRSV.apply(L, val, b)
