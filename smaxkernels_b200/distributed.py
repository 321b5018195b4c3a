"""Row-distributed SpMV, SpMM and SpGEMM over torch.distributed (one process
per GPU).

A CRS matrix is split into contiguous row blocks balanced by nonzeros; rank r
owns rows [b_r, b_{r+1}) of A and the same slice of x and y (SpMM: the same
rows of X and Y).  This is the distribution the reference's distributed
setting needs (its MPI layer is an empty file):
  * SpMV / SpMM: one exchange plus one local product.  The x slices (X row
    slices) are all-gathered into the full x (X) on every rank (NCCL over
    NVLink / NVSwitch on GPUs), then each rank runs the platform's kernel on
    its block.
  * SpGEMM: B is replicated on every rank, so each rank's rows of C = A B
    come from its rows of A alone, with no exchange; they are the same rows,
    in the same first-touch column order, as the undistributed product's.
  * SpTRSV does not shard this way and runs as independent replicas.

all_gather needs equal-sized pieces: every slice is padded to the largest one
and the padding is dropped when the full vector is assembled.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple

import numpy as np


def partition_rows(row_ptr, world: int) -> List[Tuple[int, int]]:
    """Contiguous row blocks with about nnz/world entries each: block r ends at
    the first row whose prefix count reaches (r+1)*nnz/world."""
    rp = np.asarray(row_ptr, dtype=np.int64)
    n = len(rp) - 1
    nnz = int(rp[-1])
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(rp, (r * nnz) / world, side="left")))
    cuts.append(n)
    for i in range(1, len(cuts)):  # monotone even when many rows are empty
        cuts[i] = max(cuts[i], cuts[i - 1])
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def local_block(row_ptr, col, val, rows: Tuple[int, int]):
    """The rows [b, e) of a CRS matrix as a CRS block (global column indices)."""
    b, e = rows
    rp = np.asarray(row_ptr)
    s0, s1 = int(rp[b]), int(rp[e])
    return (rp[b:e + 1] - s0).astype(np.int32), np.ascontiguousarray(col[s0:s1]), np.ascontiguousarray(val[s0:s1])


class RowDistributedSpMV:
    """y_local = (A x)[my rows] with x distributed like y.

    `blocks` is partition_rows(...) of the global matrix (the same list on
    every rank).  By default the local product is the platform's CRS SpMV
    kernel on the GPU of this rank with device-resident operands;
    `local_apply(x_full) -> y_local` replaces it (used by CPU tests of the
    exchange)."""

    def __init__(self, row_ptr_local, col_local, val_local, n_cols: int, blocks: List[Tuple[int, int]],
                 rank: int, group=None, device: Optional[str] = None,
                 local_apply: Optional[Callable] = None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.blocks = blocks
        self.rank = rank
        self.n_cols = int(n_cols)
        self.world = len(blocks)
        self.pad = max(e - b for b, e in blocks) if blocks else 0
        self.n_local = blocks[rank][1] - blocks[rank][0]
        dtype = torch.float64 if np.asarray(val_local).dtype == np.float64 else torch.float32
        self.device = torch.device(device) if device else torch.device("cpu")
        self._send = torch.zeros(self.pad, dtype=dtype, device=self.device)
        self._recv = torch.zeros(self.pad * self.world, dtype=dtype, device=self.device)
        self._x = torch.zeros(self.n_cols, dtype=dtype, device=self.device)
        self._local_apply = local_apply
        self._kernel = None
        if local_apply is None:
            from .interface import FloatType, Interface, IntType, KernelType, PlatformType
            self._smax = Interface()
            ft = FloatType.FLOAT64 if dtype == torch.float64 else FloatType.FLOAT32
            self._smax.register_kernel("spmv", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, ft)
            k = self._smax.kernel("spmv")
            self._y = torch.zeros(self.n_local, dtype=dtype, device=self.device)
            k.register_A(self.n_local, self.n_cols, len(col_local), col_local, row_ptr_local, val_local)
            k.register_B(self.n_cols, self._x)
            k.register_C(self.n_local, self._y)
            k.set_stream(torch.cuda.current_stream(self.device).cuda_stream)
            k.initialize()
            self._kernel = k

    def gather_x(self, x_local):
        """All ranks' x slices, assembled into the full x (the one exchange)."""
        n = self.n_local
        self._send[:n].copy_(x_local.reshape(-1))
        self.dist.all_gather_into_tensor(self._recv, self._send, group=self.group)
        for r, (b, e) in enumerate(self.blocks):
            self._x[b:e].copy_(self._recv[r * self.pad: r * self.pad + (e - b)])
        return self._x

    def __call__(self, x_local):
        x_full = self.gather_x(x_local)
        if self._local_apply is not None:
            return self._local_apply(x_full)
        self._kernel.apply()
        return self._y.clone()

    def close(self):
        if self._kernel is not None:
            self._smax.close()
            self._kernel = None


class RowDistributedSpMM:
    """Y_local = (A X)[my rows] for a row-major X of k columns distributed like
    Y: one all-gather of the X row slices, then the platform's row-major SpMM
    on this rank's block (or `local_apply(X_full) -> Y_local`, used by CPU
    tests of the exchange)."""

    def __init__(self, row_ptr_local, col_local, val_local, n_cols: int, k: int, blocks: List[Tuple[int, int]],
                 rank: int, group=None, device: Optional[str] = None, local_apply: Optional[Callable] = None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.blocks = blocks
        self.rank = rank
        self.k = int(k)
        self.n_cols = int(n_cols)
        self.world = len(blocks)
        self.pad = max(e - b for b, e in blocks) if blocks else 0
        self.n_local = blocks[rank][1] - blocks[rank][0]
        dtype = torch.float64 if np.asarray(val_local).dtype == np.float64 else torch.float32
        self.device = torch.device(device) if device else torch.device("cpu")
        self._send = torch.zeros(self.pad * self.k, dtype=dtype, device=self.device)
        self._recv = torch.zeros(self.pad * self.k * self.world, dtype=dtype, device=self.device)
        self._X = torch.zeros(self.n_cols * self.k, dtype=dtype, device=self.device)
        self._local_apply = local_apply
        self._kernel = None
        if local_apply is None:
            from .interface import FloatType, Interface, IntType, KernelType, PlatformType
            self._smax = Interface()
            ft = FloatType.FLOAT64 if dtype == torch.float64 else FloatType.FLOAT32
            self._smax.register_kernel("spmm", KernelType.SPMM, PlatformType.CUDA, IntType.INT32, ft)
            kern = self._smax.kernel("spmm")
            kern.set_vec_row_major(True)
            self._Y = torch.zeros(self.n_local * self.k, dtype=dtype, device=self.device)
            kern.register_A(self.n_local, self.n_cols, len(col_local), col_local, row_ptr_local, val_local)
            kern.register_B(self.n_cols, self.k, self._X)
            kern.register_C(self.n_local, self.k, self._Y)
            kern.set_stream(torch.cuda.current_stream(self.device).cuda_stream)
            kern.initialize()
            self._kernel = kern

    def gather_X(self, X_local):
        """All ranks' X row slices, assembled into the full row-major X."""
        n, k = self.n_local, self.k
        self._send[:n * k].copy_(X_local.reshape(-1))
        self.dist.all_gather_into_tensor(self._recv, self._send, group=self.group)
        for r, (b, e) in enumerate(self.blocks):
            o = r * self.pad * k
            self._X[b * k:e * k].copy_(self._recv[o:o + (e - b) * k])
        return self._X

    def __call__(self, X_local):
        X_full = self.gather_X(X_local)
        if self._local_apply is not None:
            return self._local_apply(X_full)
        self._kernel.apply()
        return self._Y.clone()

    def close(self):
        if self._kernel is not None:
            self._smax.close()
            self._kernel = None


class RowDistributedSpGEMM:
    """C_local = (A B)[my rows] with B replicated on every rank: no exchange.
    Returns (row_ptr, col, val) of this rank's rows of C (host arrays), computed
    by the platform's SpGEMM (or by `local_apply(rp, col, val) -> C rows`, used
    by CPU tests)."""

    def __init__(self, row_ptr_local, col_local, val_local, b_row_ptr, b_col, b_val, b_n_cols: int,
                 local_apply: Optional[Callable] = None):
        self._args = (np.asarray(row_ptr_local, np.int32), np.asarray(col_local, np.int32), np.asarray(val_local))
        self._b = (np.asarray(b_row_ptr, np.int32), np.asarray(b_col, np.int32), np.asarray(b_val))
        self.b_n_cols = int(b_n_cols)
        self._local_apply = local_apply

    def __call__(self):
        rp, col, val = self._args
        if self._local_apply is not None:
            return self._local_apply(rp, col, val)
        from .interface import FloatType, Interface, IntType, KernelType, PlatformType
        brp, bcol, bval = self._b
        smax = Interface()
        ft = FloatType.FLOAT64 if val.dtype == np.float64 else FloatType.FLOAT32
        smax.register_kernel("spgemm", KernelType.SPGEMM, PlatformType.CUDA, IntType.INT32, ft)
        kern = smax.kernel("spgemm")
        kern.register_A(len(rp) - 1, len(brp) - 1, len(col), col, rp, val)
        kern.register_B(len(brp) - 1, self.b_n_cols, len(bcol), bcol, brp, bval)
        kern.register_C()
        kern.run()
        _, _, _, crp, ccol, cval = kern.result()
        smax.close()
        return crp, ccol, cval


def concat_rows(parts):
    """The CRS matrix whose row blocks are `parts` (row_ptr, col, val) in rank
    order: the assembled product of RowDistributedSpGEMM."""
    rps, cols, vals, off = [np.zeros(1, np.int64)], [], [], 0
    for rp, col, val in parts:
        rps.append(np.asarray(rp[1:], np.int64) + off)
        off += int(rp[-1])
        cols.append(np.asarray(col))
        vals.append(np.asarray(val))
    return (np.concatenate(rps).astype(np.int32), np.concatenate(cols) if cols else np.zeros(0, np.int32),
            np.concatenate(vals) if vals else np.zeros(0))
