"""Row-distributed SpMV over torch.distributed (one process per GPU).

A CRS matrix is split into contiguous row blocks balanced by nonzeros; rank r
owns rows [b_r, b_{r+1}) of A and the same slice of x and y.  One product is
one exchange plus one local SpMV: the x slices are all-gathered into a full x
on every rank (NCCL over NVLink / NVSwitch on GPUs), then each rank runs the
platform's CRS SpMV on its block.  This is the exchange the reference's
distributed setting needs (its MPI layer is an empty file); SpTRSV does not
shard this way and runs as independent replicas instead.

all_gather needs equal-sized pieces: every slice is padded to the largest one
and the padding is dropped when the full x is assembled.
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
