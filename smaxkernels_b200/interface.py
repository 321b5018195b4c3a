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
import os

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
            spmv_variant=10, solve_mode=11, level_merge=12, spin_limit=13, test_force_timeout=14,
            refine=15, refine_tol=16, sweep_cluster=17, spmv_pipeline=18, timers=19)

SOLVE_AUTO, SOLVE_PER_LEVEL, SOLVE_MERGED, SOLVE_GRAPH, SOLVE_PERSISTENT, SOLVE_SYNCFREE = 0, 1, 2, 3, 4, 5


CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy: the legacy default stream as an explicit handle


def _stream_arg(stream):
    """A torch stream handle for the C ABI: 0 (the default stream) becomes cudaStreamLegacy."""
    return C.c_void_p(stream if stream else CUDA_STREAM_LEGACY)


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
        self._scs = False
        self._bcrs = False

    # -- registration -----------------------------------------------------
    def register_A(self, *args):
        """CRS (6 args), BCRS (10 args, after set_mat_bcrs) or SELL-C-sigma (13 args,
        after set_mat_scs), in the reference's argument orders (src/kernels/spmv.hpp:25-91)."""
        n = len(args)
        if self._scs:
            if n != 13:
                raise RuntimeError("SpMVKernel register_A expects 13 Sell-C-sigma args")
            (C_, sigma, n_rows, n_rows_padded, n_cols, n_chunks, n_elements, nnz, chunk_ptr, chunk_lengths, col,
             val, perm) = args
            self._keep["A"] = (chunk_ptr, chunk_lengths, col, val, perm)
            check(lib.smax_kernel_register_A_scs(self._h, int(C_), int(sigma), int(n_rows), int(n_rows_padded),
                                                 int(n_cols), int(n_chunks), int(n_elements), int(nnz),
                                                 _ptr(chunk_ptr), _ptr(chunk_lengths), _ptr(col), _ptr(val),
                                                 _ptr(perm)))
            return 0
        if self._bcrs:
            if n != 10:
                raise RuntimeError("SpMVKernel register_A expects 10 BCRS args")
            n_rows, n_cols, n_blocks, bh, bw, hpad, wpad, col, row_ptr, val = args
            self._keep["A"] = (col, row_ptr, val)
            check(lib.smax_kernel_register_A_bcrs(self._h, int(n_rows), int(n_cols), int(n_blocks), int(bh),
                                                  int(bw), int(hpad), int(wpad), _ptr(col), _ptr(row_ptr),
                                                  _ptr(val)))
            return 0
        if n == 6:
            n_rows, n_cols, nnz, col, row_ptr, val = args
            self._keep["A"] = (col, row_ptr, val)
            check(lib.smax_kernel_register_A_crs(self._h, int(n_rows), int(n_cols), int(nnz), _ptr(col),
                                                 _ptr(row_ptr), _ptr(val)))
            return 0
        raise RuntimeError(f"{self.kernel_type.name} register_A expects 6 args")

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
        if self.kernel_type == KernelType.SPGEMM:
            if len(args) != 6:
                raise RuntimeError("SpGEMMKernel register_B expects 6 args")
            n_rows, n_cols, nnz, col, row_ptr, val = args
            self._keep["B"] = (col, row_ptr, val)
            check(lib.smax_kernel_register_B_crs(self._h, int(n_rows), int(n_cols), int(nnz), _ptr(col),
                                                 _ptr(row_ptr), _ptr(val)))
            return 0
        return self._register_dense(1, args)

    def register_C(self, *args):
        if self.kernel_type == KernelType.SPGEMM:
            if len(args) != 0:
                raise RuntimeError("SpGEMMKernel register_C takes no arguments here: read the result with "
                                   "result() after run(); the references are owned by the kernel")
            self._cref = [C.c_uint64(0), C.c_uint64(0), C.c_uint64(0), C.c_void_p(), C.c_void_p(), C.c_void_p()]
            r = self._cref
            check(lib.smax_kernel_register_C_crs_ref(self._h, C.byref(r[0]), C.byref(r[1]), C.byref(r[2]),
                                                     C.byref(r[3]), C.byref(r[4]), C.byref(r[5])))
            return 0
        return self._register_dense(2, args)

    def result(self):
        """SpGEMM: C as (n_rows, n_cols, nnz, row_ptr, col, val) numpy copies of
        the arrays finalize() allocated (which are then released)."""
        r = self._cref
        n_rows, n_cols, nnz = r[0].value, r[1].value, r[2].value
        vt = np.float64 if self.float_type == FloatType.FLOAT64 else np.float32
        return (n_rows, n_cols, nnz, _take(r[4].value, n_rows + 1, np.int32), _take(r[3].value, nnz, np.int32),
                _take(r[5].value, nnz, vt))

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
        self._scs = bool(v)
        return self._flag("mat_scs", v)

    def set_mat_bcrs(self, v):
        self._bcrs = bool(v)
        return self._flag("mat_bcrs", v)

    def set_block_column_major(self, v):
        return self._flag("block_column_major", v)

    def set_kernel_implementation(self, impl):
        return self._flag("kernel_impl", int(impl))

    def set_spmv_variant(self, v: int):
        """CRS SpMV kernel: 0 auto, 1 warp-stream, 2 row-tile.  Row-major SpMM:
        0 auto, 1 a grid of all rows, 2 one CTA per SM walking a row range."""
        return self._flag("spmv_variant", v)

    def set_timers(self, on: bool):
        """CUDA-event stopwatches around every apply (the "apply" timer and
        SpGEMM's phases; default on).  Off, applies record no events: a
        timing event between launches costs about 2.5 us of device time,
        which matters for small matrices in a loop."""
        return self._flag("timers", int(bool(on)))

    def set_spmv_pipeline(self, blocks: int):
        """CRS SpMV with host operands: row blocks whose part of y is downloaded
        while later blocks compute; block b holds 2^b / (2^B - 1) of the entries
        (default 6, at most 16 used; 0 or 1: off)."""
        return self._flag("spmv_pipeline", blocks)

    def set_solve_mode(self, mode: int):
        """SpTRSV/SpTRSM launch scheme: SOLVE_AUTO, SOLVE_PER_LEVEL, SOLVE_MERGED, SOLVE_GRAPH,
        SOLVE_PERSISTENT or SOLVE_SYNCFREE."""
        return self._flag("solve_mode", mode)

    def set_spin_limit(self, kilo_polls: int):
        """Polls (x 1000) before a wait of the persistent or sync-free solve gives up with TIMEOUT."""
        return self._flag("spin_limit", kilo_polls)

    def set_sweep_cluster(self, v: bool):
        """SpTRSV: let runs with levels wider than 1024 rows use a thread-block cluster."""
        return self._flag("sweep_cluster", int(bool(v)))

    def set_level_merge(self, rows: int):
        """Levels with at most `rows` (row, right-hand side) pairs run merged in one CTA."""
        return self._flag("level_merge", rows)

    def mark_A_dirty(self):
        return self._flag("a_dirty", 1)

    def swap_operands(self):
        """x <-> y (src/kernels/spmv.hpp:197-200): the registered B and C, and
        their device copies, exchange roles."""
        check(lib.smax_kernel_swap_operands(self._h))
        kb, kc = self._keep.get("B"), self._keep.get("C")
        self._keep["B"], self._keep["C"] = kc, kb
        return 0

    def set_refine(self, steps: int, tol_exp: int = 0):
        """float64 SpTRSV: solve in FP32 and apply `steps` FP64-residual
        corrections; with tol_exp > 0 stop once max|dx| <= 10^-tol_exp max|x|."""
        self._flag("refine", steps)
        return self._flag("refine_tol", tol_exp)

    def refine_stats(self):
        """(corrections applied, max|dx|/max|x| of the last one) of the last refined solve."""
        n, r = C.c_int(0), C.c_double(0.0)
        check(lib.smax_kernel_get_refine_stats(self._h, C.byref(n), C.byref(r)))
        return n.value, r.value

    # -- reverse mode -----------------------------------------------------
    def _same_space(self, *arrs):
        dev = bool(self._device)
        for a in arrs:
            if a is not None and _is_torch_cuda(a) != dev:
                raise RuntimeError("adjoint operands must live where B and C were registered "
                                   f"({'device tensors' if dev else 'host arrays'})")

    def adjoint(self, g, d_in=None, d_val=None, x=None):
        """Reverse mode of an initialized CRS SpMV or SpTRSV kernel for the loss
        gradient g: d_in = A^T g (SpMV) or lambda = L^-T g (SpTRSV, = dLoss/db);
        d_val = g[row] x[col] (SpMV) or -lambda[row] x[col] (SpTRSV) in the
        device copy's entry order; x defaults to the registered B."""
        self._same_space(g, d_in, d_val, x)
        check(lib.smax_kernel_adjoint(self._h, _ptr(x), _ptr(g), _ptr(d_in), _ptr(d_val)))
        return 0

    def update_A_values(self, val):
        """New values for the device copy of A (same pattern and entry order)."""
        self._same_space(val)
        check(lib.smax_kernel_update_A_values(self._h, _ptr(val)))
        return 0

    # -- tuning -----------------------------------------------------------
    def autotune(self) -> dict:
        """Times the launch variants on the registered operands, keeps the
        fastest (cached per matrix for the process) and returns the choice."""
        t = _lib.Tuning()
        check(lib.smax_kernel_autotune(self._h, C.byref(t)))
        return _lib.struct_dict(t)

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
        """Launch on the caller's CUDA stream, e.g. torch.cuda.current_stream().cuda_stream.
        0 (torch's default stream) means the legacy default stream; None
        restores the kernel's own stream."""
        if stream_ptr is None:
            arg = None
        else:
            arg = C.c_void_p(stream_ptr if stream_ptr else CUDA_STREAM_LEGACY)
        check(lib.smax_kernel_set_stream(self._h, arg))

    def _destroy(self):
        if self._h:
            lib.smax_kernel_destroy(self._h)
            self._h = None


class TriangularBatch:
    """Batched SpTRSV over independent lower-triangular matrices (C ABI
    smax_batch_sptrsv_*): one persistent kernel with a device work queue."""

    def __init__(self, mats, float_type: FloatType = FloatType.FLOAT64):
        """mats: list of (row_ptr, col, val) numpy CRS arrays (square, with diagonal)."""
        n = len(mats)
        self._keep = [(_i32(rp), _i32(c), np.ascontiguousarray(v)) for rp, c, v in mats]
        nr = (C.c_uint64 * n)(*[len(m[0]) - 1 for m in self._keep])
        nz = (C.c_uint64 * n)(*[len(m[1]) for m in self._keep])
        rps = (C.c_void_p * n)(*[m[0].ctypes.data for m in self._keep])
        cls = (C.c_void_p * n)(*[m[1].ctypes.data for m in self._keep])
        vls = (C.c_void_p * n)(*[m[2].ctypes.data for m in self._keep])
        h = C.c_void_p()
        check(lib.smax_batch_sptrsv_create(C.byref(h), int(float_type), n, nr, nz, rps, cls, vls))
        self._h = h
        self.n_mats = n

    def row_offset(self, m: int) -> int:
        return int(lib.smax_batch_row_offset(self._h, m))

    def info(self):
        nr, tl, ml = C.c_uint64(0), C.c_int(0), C.c_int(0)
        check(lib.smax_batch_info(self._h, C.byref(nr), C.byref(tl), C.byref(ml)))
        return nr.value, tl.value, ml.value

    def solve(self, rhs, x, mode: int = 0, stream: int = 0):
        """rhs, x: CUDA tensors of the packed rows; stream: a torch stream handle
        (0, the default, is torch's default stream)."""
        check(lib.smax_batch_sptrsv_solve(self._h, _ptr(rhs), _ptr(x), int(mode), _stream_arg(stream)))

    def close(self):
        if self._h:
            lib.smax_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _ftype(dtype) -> int:
    if np.dtype(dtype) == np.float64:
        return int(FloatType.FLOAT64)
    if np.dtype(dtype) == np.float32:
        return int(FloatType.FLOAT32)
    raise TypeError("values must be float32 or float64")


def _take(p, n, dtype):
    """Copies n elements of a library-allocated host array into numpy and frees it."""
    if not p:
        return np.zeros(0, dtype)
    out = np.empty(n, dtype=dtype)
    if n:
        C.memmove(out.ctypes.data, p, n * out.itemsize)
    lib.smax_free_host(p)
    return out


class Utils:
    """SMAX::Utils (src/utils.hpp:12-87): the work runs on the GPU; inputs and
    outputs are host numpy arrays, as the reference's are host arrays."""

    def __init__(self, iface: "Interface"):
        self._iface = iface

    def tune_spmv_format(self, n_rows, n_cols, nnz, col, row_ptr, val) -> dict:
        """Times CRS (both kernels), SELL-C-sigma and BCRS candidates of this
        matrix on the GPU and returns the fastest (smax_utils_tune_spmv_format)."""
        col, row_ptr = _i32(col), _i32(row_ptr)
        val = np.ascontiguousarray(val)
        ft = FloatType.FLOAT64 if val.dtype == np.float64 else FloatType.FLOAT32
        out = _lib.FormatChoice()
        check(lib.smax_utils_tune_spmv_format(int(ft), int(n_rows), int(n_cols), int(nnz), _ptr(row_ptr),
                                              _ptr(col), _ptr(val), C.byref(out)))
        d = _lib.struct_dict(out)
        d["format_name"] = ("CRS", "SELL-C-sigma", "BCRS")[d["format"]]
        return d

    def convert_crs_to_scs(self, n_rows, n_cols, nnz, col, row_ptr, val, C_, sigma) -> dict:
        """Returns the 13 SELL-C-sigma fields of convert_crs_to_scs as a dict."""
        col, row_ptr = _i32(col), _i32(row_ptr)
        val = np.ascontiguousarray(val)
        meta = (C.c_uint64 * 6)()
        ptrs = [C.c_void_p() for _ in range(5)]
        check(lib.smax_utils_convert_crs_to_scs(int(IntType.INT32), _ftype(val.dtype), int(n_rows), int(n_cols),
                                                int(nnz), _ptr(col), _ptr(row_ptr), _ptr(val), int(C_),
                                                int(sigma), meta, *[C.byref(p) for p in ptrs]))
        nr, npad, nc, nch, ne, nz = (int(v) for v in meta)
        return dict(C=int(C_), sigma=int(sigma), n_rows=nr, n_rows_padded=npad, n_cols=nc, n_chunks=nch,
                    n_elements=ne, nnz=nz, chunk_ptr=_take(ptrs[0].value, nch + 1, np.int32),
                    chunk_lengths=_take(ptrs[1].value, nch, np.int32), col=_take(ptrs[2].value, ne, np.int32),
                    val=_take(ptrs[3].value, ne, val.dtype), perm=_take(ptrs[4].value, nr, np.int32))

    def convert_crs_to_bcrs(self, n_rows, n_cols, nnz, col, row_ptr, val, b_height, b_width, height_pad,
                            width_pad, block_column_major) -> dict:
        col, row_ptr = _i32(col), _i32(row_ptr)
        val = np.ascontiguousarray(val)
        meta = (C.c_uint64 * 7)()
        ptrs = [C.c_void_p() for _ in range(3)]
        check(lib.smax_utils_convert_crs_to_bcrs(int(IntType.INT32), _ftype(val.dtype), int(n_rows), int(n_cols),
                                                 int(nnz), _ptr(col), _ptr(row_ptr), _ptr(val), int(b_height),
                                                 int(b_width), int(height_pad), int(width_pad),
                                                 int(bool(block_column_major)), meta,
                                                 *[C.byref(p) for p in ptrs]))
        nr, nc, nb, bh, bw, hp, wp = (int(v) for v in meta)
        return dict(n_rows=nr, n_cols=nc, n_blocks=nb, b_height=bh, b_width=bw, height_pad=hp, width_pad=wp,
                    col=_take(ptrs[0].value, nb, np.int32), row_ptr=_take(ptrs[1].value, nr + 1, np.int32),
                    val=_take(ptrs[2].value, nb * hp * wp, val.dtype))


    # -- level sets and permutations (src/utils/permutations.hpp) --------------
    def print_timers(self, file=None):
        """Utils::print_timers (src/utils.hpp:24): every registered kernel's
        initialize / apply / finalize stopwatches and their total (SpGEMM also
        its phases), in seconds."""
        import sys
        out = file or sys.stdout
        for name, k in self._iface._kernels.items():
            parts = ["initialize", "apply", "finalize"]
            t = {p: k.timer(p) for p in parts}
            print(f"+{'-' * 19} SMAX Timer {'-' * 19}+", file=out)
            print(f"Total time in '{name}': {sum(t.values()):.3e} [s]", file=out)
            for p_ in parts:
                print(f"| {p_.capitalize()} time: {t[p_]:.3e} [s]", file=out)
            if k.kernel_type == KernelType.SPGEMM:
                for p_ in ("Symbolic_Setup", "Fused_Gustavson", "Alloc_C", "Compress"):
                    print(f"|   {p_}: {k.timer(p_):.3e} [s]", file=out)
            print(f"+{'-' * 50}+", file=out)

    def read_mtx(self, path: str, dtype=np.float64):
        """A Matrix Market file as CRS (n_rows, n_cols, nnz, row_ptr, col, val),
        read as the reference's examples read it (smax_utils_read_mtx)."""
        nr, nc, nz = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
        ptrs = [C.c_void_p() for _ in range(3)]
        check(lib.smax_utils_read_mtx(os.fsencode(path), _ftype(np.dtype(dtype)), C.byref(nr), C.byref(nc),
                                      C.byref(nz), *[C.byref(p) for p in ptrs]))
        n, m, z = nr.value, nc.value, nz.value
        return (n, m, z, _take(ptrs[0].value, n + 1, np.int32), _take(ptrs[1].value, z, np.int32),
                _take(ptrs[2].value, z, np.dtype(dtype)))

    def convert_coo_to_crs(self, n_rows, n_cols, I, J, val, dtype=np.float64):
        """COO (0-based) to CRS, entries stably sorted by row (file order kept
        within a row): (row_ptr, col, val)."""
        I, J = _i32(I), _i32(J)
        val = np.ascontiguousarray(val, dtype=np.float64)
        ptrs = [C.c_void_p() for _ in range(3)]
        check(lib.smax_utils_convert_coo_to_crs(_ftype(np.dtype(dtype)), int(n_rows), int(n_cols), len(I), _ptr(I),
                                                _ptr(J), _ptr(val), *[C.byref(p) for p in ptrs]))
        return (_take(ptrs[0].value, int(n_rows) + 1, np.int32), _take(ptrs[1].value, len(I), np.int32),
                _take(ptrs[2].value, len(I), np.dtype(dtype)))

    def build_symmetric_crs(self, row_ptr, col, n_rows):
        """Pattern of A + A^T: returns (sym_row_ptr, sym_col, sym_nnz)."""
        row_ptr, col = _i32(row_ptr), _i32(col)
        pr, pc, nz = C.c_void_p(), C.c_void_p(), C.c_uint64(0)
        check(lib.smax_utils_build_symmetric_crs(int(IntType.INT32), int(n_rows), _ptr(row_ptr), _ptr(col),
                                                 C.byref(pr), C.byref(pc), C.byref(nz)))
        return _take(pr.value, int(n_rows) + 1, np.int32), _take(pc.value, nz.value, np.int32), nz.value

    def generate_perm(self, n_rows, row_ptr, col, perm, inv_perm, type_="BFS"):
        """Fills perm / inv_perm (int32 arrays of n_rows) and stores the level
        pointer in the Interface (get_n_levels / get_level_ptr_at)."""
        for a in (perm, inv_perm):
            if not (isinstance(a, np.ndarray) and a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]):
                raise TypeError("perm and inv_perm must be C-contiguous int32 numpy arrays")
        row_ptr, col = _i32(row_ptr), _i32(col)
        check(lib.smax_utils_generate_perm(self._iface._ctx, int(IntType.INT32), int(n_rows), _ptr(row_ptr),
                                           _ptr(col), _ptr(perm), _ptr(inv_perm), type_.encode()))

    def sanity_check_perm(self, n_rows, row_ptr, col, colors) -> bool:
        """Utils::sanity_check_perm: no row shares a non-zero colour with a
        lower neighbour."""
        valid, bad = C.c_int(0), C.c_int64(-1)
        check(lib.smax_utils_sanity_check_perm(int(IntType.INT32), int(n_rows), _ptr(_i32(row_ptr)), _ptr(_i32(col)),
                                               _ptr(_i32(colors)), C.byref(valid), C.byref(bad)))
        return bool(valid.value)

    def apply_mat_perm(self, n_rows, row_ptr, col, val, perm_row_ptr, perm_col, perm_val, perm, inv_perm):
        row_ptr, col, perm, inv_perm = _i32(row_ptr), _i32(col), _i32(perm), _i32(inv_perm)
        val = np.ascontiguousarray(val)
        check(lib.smax_utils_apply_mat_perm(int(IntType.INT32), _ftype(val.dtype), int(n_rows), _ptr(row_ptr),
                                            _ptr(col), _ptr(val), _ptr(perm_row_ptr), _ptr(perm_col),
                                            _ptr(perm_val), _ptr(perm), _ptr(inv_perm)))

    def apply_vec_perm(self, n_rows, vec, vec_perm, perm):
        perm = _i32(perm)
        vec = np.ascontiguousarray(vec)
        check(lib.smax_utils_apply_vec_perm(_ftype(vec.dtype), int(n_rows), _ptr(vec), _ptr(vec_perm), _ptr(perm)))

    def level_aware_copy(self, src_row_ptr, dest_row_ptr, src_col, dest_col, src_val, dest_val):
        """src/utils/permutations.hpp:876-897: a first-touch (NUMA) copy on the
        CPU platform; on this platform a plain copy of the three arrays."""
        dest_row_ptr[...] = src_row_ptr
        dest_col[...] = src_col
        dest_val[...] = src_val


class Interface:
    """SMAX::Interface for the CUDA platform (src/interface.hpp:21-48)."""

    def __init__(self):
        h = C.c_void_p()
        check(lib.smax_ctx_create(C.byref(h)))
        self._ctx = h
        self._kernels: dict[str, Kernel] = {}
        self.utils = Utils(self)

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

    def set_levels(self, lvl_ptr):
        """Stores a level pointer computed elsewhere (n_levels + 1 entries)."""
        lp = np.ascontiguousarray(lvl_ptr, dtype=np.int32)
        check(lib.smax_ctx_set_levels(self._ctx, len(lp) - 1, _ptr(lp)))

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
