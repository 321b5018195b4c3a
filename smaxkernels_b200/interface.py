"""Python mirror of the SmaxKernels ``SMAX::Interface`` API over the C ABI.

Same names, argument order and meaning as the reference
(src/interface.hpp:21-48, src/kernel.hpp:7-127, src/kernels/*.hpp), so a test
written against the reference reads the same here::

    smax = Interface()
    smax.register_kernel("my_spmv", KernelType.SPMV, PlatformType.CUDA)
    smax.kernel("my_spmv").register_A(n_rows, n_cols, nnz, col, row_ptr, val)
    smax.kernel("my_spmv").register_B(n_cols, x)
    smax.kernel("my_spmv").register_C(n_rows, y)
    smax.kernel("my_spmv").run()

Arrays are numpy arrays (host memory, as in the reference) or CUDA tensors of
torch (device memory; the kernel then gets SMAX_FLAG_DEVICE_POINTERS).  Only
PlatformType.CUDA exists on this platform; the reference's CPU path is not
re-implemented.  Errors raise SmaxError (the reference throws
std::runtime_error from ErrorHandler::fatal, src/error_handler.cpp:92-96).
"""
from __future__ import annotations

import ctypes as C
import enum

import numpy as np

from . import _lib
from ._lib import check, lib


class KernelType(enum.IntEnum):
    SPMV = 0
    SPMM = 1
    SPGEMM = 2
    SPTRSV = 3
    SPTRSM = 4


class PlatformType(enum.IntEnum):
    CPU = 0
    CUDA = 1


class IntType(enum.IntEnum):
    INT16 = 0
    INT32 = 1
    INT64 = 2
    UINT16 = 3
    UINT32 = 4
    UINT64 = 5


class FloatType(enum.IntEnum):
    FLOAT32 = 0
    FLOAT64 = 1


class SpMVType(enum.IntEnum):
    naive_thread_per_row = 0
    naive_warp_group = 1
    naive_warp_shuffle = 2


FLAG = dict(mat_perm=0, mat_upper_triang=1, mat_lower_triang=2, vec_row_major=3, mat_scs=4, mat_bcrs=5,
            block_column_major=6, kernel_impl=7, device_pointers=8, a_dirty=9,
            spmv_variant=10)


def _is_torch_cuda(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


def _ptr(a):
    """Address of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return C.c_void_p(a.ctypes.data)
    raise TypeError(f"unsupported array type {type(a)}")


class Kernel:
    """One registered kernel (src/kernel.hpp:7-127)."""

    def __init__(self, iface: "Interface", name: str, handle: C.c_void_p, ktype: KernelType, itype: IntType,
                 ftype: FloatType):
        self._iface = iface
        self.name = name
        self._h = handle
        self.kernel_type = ktype
        self.int_type = itype
        self.float_type = ftype
        self._keep = {}  # registered arrays stay alive while registered
        self._device = None

    # -- registration -----------------------------------------------------
    def register_A(self, *args):
        n = len(args)
        if n == 6:
            n_rows, n_cols, nnz, col, row_ptr, val = args
            self._keep["A"] = (col, row_ptr, val)
            check(lib.smax_kernel_register_A_crs(self._h, int(n_rows), int(n_cols), int(nnz), _ptr(col),
                                                 _ptr(row_ptr), _ptr(val)))
            return 0
        raise RuntimeError(f"{self.kernel_type.name} register_A: unsupported argument count {n}")

    def _register_dense(self, slot: int, args):
        if len(args) == 2:
            n_rows, arr = args
            n_cols = 1
        elif len(args) == 3:
            n_rows, n_cols, arr = args
        else:
            raise RuntimeError(f"{self.kernel_type.name} register_{'B' if slot == 1 else 'C'}: bad argument count")
        dev = _is_torch_cuda(arr)
        if self._device is None:
            self._device = dev
            check(lib.smax_kernel_set_flag(self._h, FLAG["device_pointers"], int(dev)))
        elif self._device != dev:
            raise RuntimeError("B and C must both be host arrays or both device tensors")
        self._keep["B" if slot == 1 else "C"] = arr
        check(lib.smax_kernel_register_dense(self._h, slot, int(n_rows), int(n_cols), _ptr(arr)))
        return 0

    def register_B(self, *args):
        return self._register_dense(1, args)

    def register_C(self, *args):
        return self._register_dense(2, args)

    # -- flags ------------------------------------------------------------
    def _flag(self, name, v):
        check(lib.smax_kernel_set_flag(self._h, FLAG[name], int(v)))
        return 0

    def set_mat_perm(self, v):
        return self._flag("mat_perm", v)

    def set_mat_upper_triang(self, v):
        return self._flag("mat_upper_triang", v)

    def set_mat_lower_triang(self, v):
        return self._flag("mat_lower_triang", v)

    def set_vec_row_major(self, v):
        return self._flag("vec_row_major", v)

    def set_mat_scs(self, v):
        return self._flag("mat_scs", v)

    def set_mat_bcrs(self, v):
        return self._flag("mat_bcrs", v)

    def set_block_column_major(self, v):
        return self._flag("block_column_major", v)

    def set_kernel_implementation(self, impl):
        return self._flag("kernel_impl", int(impl))

    def set_spmv_variant(self, v: int):
        """CRS SpMV kernel: 0 auto, 1 warp-stream, 2 row-tile."""
        return self._flag("spmv_variant", v)

    def mark_A_dirty(self):
        return self._flag("a_dirty", 1)

    # -- execution --------------------------------------------------------
    def initialize(self, A_offset=0, B_offset=0, C_offset=0):
        check(lib.smax_kernel_initialize(self._h, A_offset, B_offset, C_offset))
        return 0

    def apply(self, A_offset=0, B_offset=0, C_offset=0):
        check(lib.smax_kernel_apply(self._h, A_offset, B_offset, C_offset))
        return 0

    def finalize(self, A_offset=0, B_offset=0, C_offset=0):
        check(lib.smax_kernel_finalize(self._h, A_offset, B_offset, C_offset))
        return 0

    def run(self, A_offset=0, B_offset=0, C_offset=0):
        check(lib.smax_kernel_run(self._h, A_offset, B_offset, C_offset))
        return 0

    def sync(self):
        check(lib.smax_kernel_sync(self._h))

    def timer(self, name: str) -> float:
        s = C.c_double(0.0)
        check(lib.smax_kernel_get_timer(self._h, name.encode(), C.byref(s)))
        return s.value

    @property
    def stream(self) -> int:
        return lib.smax_kernel_stream(self._h) or 0

    def set_stream(self, stream_ptr: int | None):
        """Launch on the caller's CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        check(lib.smax_kernel_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def _destroy(self):
        if self._h:
            lib.smax_kernel_destroy(self._h)
            self._h = None


class Interface:
    """SMAX::Interface for the CUDA platform (src/interface.hpp:21-48)."""

    def __init__(self):
        h = C.c_void_p()
        check(lib.smax_ctx_create(C.byref(h)))
        self._ctx = h
        self._kernels: dict[str, Kernel] = {}

    def register_kernel(self, name: str, kernel_type: KernelType, platform: PlatformType = PlatformType.CUDA,
                        int_type: IntType = IntType.INT32, float_type: FloatType = FloatType.FLOAT64) -> int:
        if platform != PlatformType.CUDA:
            raise RuntimeError("this platform implements PlatformType.CUDA only")
        h = C.c_void_p()
        check(lib.smax_kernel_create(C.byref(h), self._ctx, int(kernel_type), int(int_type), int(float_type)))
        if name in self._kernels:
            self._kernels[name]._destroy()
        self._kernels[name] = Kernel(self, name, h, KernelType(kernel_type), IntType(int_type),
                                     FloatType(float_type))
        return 0

    def kernel(self, name: str) -> Kernel:
        try:
            return self._kernels[name]
        except KeyError:
            raise RuntimeError(f"[FATAL] Kernel: '{name}' does not exist.") from None

    def get_n_levels(self) -> int:
        return lib.smax_ctx_get_n_levels(self._ctx)

    def get_level_ptr_at(self, idx: int) -> int:
        return lib.smax_ctx_get_level_ptr_at(self._ctx, idx)

    def close(self):
        for k in self._kernels.values():
            k._destroy()
        self._kernels.clear()
        if self._ctx:
            lib.smax_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
