"""CPU-only checks of the drop-in boundary: the C-ABI library loads, exports
every function include/*.h declares, and fails cleanly (status code, message)
when no GPU is present.  No compute call is made here."""
import ctypes
import glob
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(smax_\w+)\s*\(", src, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_functions():
    names = declared_functions()
    assert "smax_kernel_run" in names and "smax_abi_version" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    from smaxkernels_b200 import _lib
    missing = [n for n in declared_functions() if not hasattr(_lib.lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_table_matches_header():
    from smaxkernels_b200 import _lib
    assert set(_lib.SIGNATURES) == set(declared_functions())


def test_abi_version():
    from smaxkernels_b200 import _lib
    assert _lib.lib.smax_abi_version() == 1


def test_no_gpu_is_an_error_not_a_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from smaxkernels_b200 import _lib
    ctx = ctypes.c_void_p()
    assert _lib.lib.smax_ctx_create(ctypes.byref(ctx)) == 0
    k = ctypes.c_void_p()
    rc = _lib.lib.smax_kernel_create(ctypes.byref(k), ctx, 0, 1, 1)
    assert rc == _lib.ERR_CUDA
    assert _lib.lib.smax_last_error()
    assert _lib.lib.smax_ctx_destroy(ctx) == 0


def test_unsupported_types_rejected_before_any_cuda_call():
    from smaxkernels_b200 import _lib
    k = ctypes.c_void_p()
    assert _lib.lib.smax_kernel_create(ctypes.byref(k), None, 0, 2, 1) == _lib.ERR_UNSUPPORTED_TYPE  # int64
    assert _lib.lib.smax_kernel_create(ctypes.byref(k), None, 9, 1, 1) == _lib.ERR_BAD_ARG
    assert b"int32" in _lib.lib.smax_last_error() or _lib.lib.smax_last_error()


def test_python_interface_unknown_kernel_is_fatal():
    from smaxkernels_b200 import Interface
    smax = Interface()
    with pytest.raises(RuntimeError, match="does not exist"):
        smax.kernel("nope")
    smax.close()


def test_product_does_not_import_oracle():
    """The product package never routes through the CPU checkers."""
    for f in glob.glob(os.path.join(REPO, "smaxkernels_b200", "**", "*.py"), recursive=True):
        src = open(f).read()
        assert "oracle" not in re.sub(r"#.*|\"\"\"[\s\S]*?\"\"\"", "", src), f


def test_ctx_set_levels_validates_and_stores():
    """A level pointer computed elsewhere (the reference's CPU generate_perm)
    is stored in the context; malformed ones are rejected."""
    from smaxkernels_b200 import _lib
    ctx = ctypes.c_void_p()
    assert _lib.lib.smax_ctx_create(ctypes.byref(ctx)) == 0
    lp = (ctypes.c_int * 4)(0, 3, 3, 10)
    assert _lib.lib.smax_ctx_set_levels(ctx, 3, lp) == 0
    assert _lib.lib.smax_ctx_get_n_levels(ctx) == 3
    assert [_lib.lib.smax_ctx_get_level_ptr_at(ctx, i) for i in range(4)] == [0, 3, 3, 10]
    bad = (ctypes.c_int * 3)(0, 5, 4)
    assert _lib.lib.smax_ctx_set_levels(ctx, 2, bad) == _lib.ERR_BAD_ARG
    bad0 = (ctypes.c_int * 2)(1, 4)
    assert _lib.lib.smax_ctx_set_levels(ctx, 1, bad0) == _lib.ERR_BAD_ARG
    assert _lib.lib.smax_ctx_get_n_levels(ctx) == 3  # unchanged by the rejected calls
    assert _lib.lib.smax_ctx_destroy(ctx) == 0


def test_python_flag_table_matches_header():
    """interface.FLAG names every SMAX_FLAG_* of the header with its value."""
    from smaxkernels_b200.interface import FLAG
    src = open(os.path.join(REPO, "include", "smax_b200.h")).read()
    header = {m.group(1).lower(): int(m.group(2)) for m in re.finditer(r"#define SMAX_FLAG_(\w+) (\d+)", src)}
    assert header == FLAG
