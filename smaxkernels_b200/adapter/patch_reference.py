"""Adds the B200 platform to a SmaxKernels checkout and builds its unit tests on it.

    python smaxkernels_b200/adapter/patch_reference.py [--ref-root DIR] [--out DIR] [--build] [--diff]

1. Copies the checkout's src/ to OUT/include/SmaxKernels (the install layout
   its examples include) and applies the edits below, each at an anchor that
   must occur exactly once; the checkout itself is never written.
2. --diff prints the edits as a unified diff against the checkout.
3. --build generates the reference's own test runner (examples/tests: its
   run_tests.cpp.in with every test header, as its CMake does) and compiles it
   with the patched library sources, SMAX_B200_MODE=1 (the CUDA arms call this
   library, smax_b200_platform.hpp) and SMAX_B200_ROUTE_ALL=1 (every kernel
   registered, whatever platform the test names, runs on the B200 platform),
   linked against smaxkernels_b200/libsmax_b200.so.  The runner is
   OUT/run_tests (OUT defaults to smaxkernels_b200/adapter/_build, git-ignored);
   run it on a GPU machine.

The edits (file: what):
  common.hpp        KernelContext holds the platform's per-kernel state and
                    releases it; the platform header is included at the end
  kernels/spmv/spmv_cuda.hpp
                    initialize_cuda / apply_cuda / finalize_cuda call B200::spmv
  kernels/spmm.hpp, spgemm.hpp, sptrsv.hpp, sptrsm.hpp
                    the dispatcher gains a PlatformType::CUDA arm
  interface.cpp     PlatformType::CUDA is accepted in a B200 build, and with
                    SMAX_B200_ROUTE_ALL every kernel is registered on it
Without SMAX_B200_MODE the patched sources compile to the reference as it was.
"""
from __future__ import annotations

import argparse
import difflib
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(REPO, "smaxkernels_b200", "libsmax_b200.so")

_B200_CTX = """#if SMAX_B200_MODE
    // state of the B200 platform for this kernel (smax_b200_platform.hpp)
    void *b200 = nullptr;
    ~KernelContext();
    KernelContext(const KernelContext &) = delete;
    KernelContext &operator=(const KernelContext &) = delete;
#endif
"""

_INCLUDE_PLATFORM = """
#if SMAX_B200_MODE
#include "smax_b200_platform.hpp"
#endif
"""


def _spmv_arm(phase: str) -> str:
    return ("#if SMAX_B200_MODE\n"
            f"    return B200::spmv(B200::Phase::{phase}, k_ctx, args, flags, A_offset, x_offset, y_offset);\n"
            "#endif\n")


def _dispatch_arm(call: str) -> str:
    return ("#if SMAX_B200_MODE\n"
            "        case PlatformType::CUDA:\n"
            f"            return {call};\n"
            "#endif\n")


_NOT_SUPPORTED = '        default:\n            std::cerr << "Error: Platform not supported\\n";'

# (file, anchor, text, where): where is "after" or "before" the anchor, or
# "replace" it with text
EDITS = [
    ("common.hpp", "        : kernel_type(kt), platform_type(pt), int_type(it), float_type(ft) {}\n", _B200_CTX,
     "after"),
    ("common.hpp", None, _INCLUDE_PLATFORM, "append"),
    ("kernels/spmv/spmv_cuda.hpp",
     "int initialize_cuda(Timers *timers, KernelContext *k_ctx, Args *args,\n"
     "                    Flags *flags, ULL A_offset, ULL x_offset, ULL y_offset) {\n", _spmv_arm("Initialize"),
     "after"),
    ("kernels/spmv/spmv_cuda.hpp",
     "int apply_cuda(Timers *timers, KernelContext *k_ctx, Args *args, Flags *flags,\n"
     "               ULL A_offset, ULL x_offset, ULL y_offset) {\n", _spmv_arm("Apply"), "after"),
    ("kernels/spmv/spmv_cuda.hpp",
     "int finalize_cuda(Timers *timers, KernelContext *k_ctx, Args *args,\n"
     "                  Flags *flags, ULL A_offset, ULL x_offset, ULL y_offset) {\n", _spmv_arm("Finalize"),
     "after"),
    ("kernels/spmm.hpp", _NOT_SUPPORTED,
     _dispatch_arm("B200::spmm(B200::phase_of(label), k_ctx.get(), args.get(), flags.get(), A_offset, "
                   "X_offset, Y_offset)"), "before"),
    ("kernels/spgemm.hpp", _NOT_SUPPORTED,
     _dispatch_arm("B200::spgemm(B200::phase_of(label), k_ctx.get(), args.get(), flags.get())"), "before"),
    ("kernels/sptrsv.hpp", _NOT_SUPPORTED,
     _dispatch_arm("B200::sptrsv(B200::phase_of(label), k_ctx.get(), args.get(), flags.get())"), "before"),
    ("kernels/sptrsm.hpp", _NOT_SUPPORTED,
     _dispatch_arm("B200::sptrsm(B200::phase_of(label), k_ctx.get(), args.get(), flags.get())"), "before"),
    ("interface.cpp", "#if !SMAX_CUDA_MODE\n    if (platform == PlatformType::CUDA)",
     "#if !SMAX_CUDA_MODE && !SMAX_B200_MODE\n    if (platform == PlatformType::CUDA)", "replace"),
    ("interface.cpp", "    std::unique_ptr<KernelContext> k_ctx = std::make_unique<KernelContext>(",
     "#if SMAX_B200_MODE && SMAX_B200_ROUTE_ALL\n"
     "    platform = PlatformType::CUDA;  // every kernel on the B200 platform\n"
     "#endif\n", "before"),
]

CONFIG = ("#pragma once\n#define SMAX_VERSION_MAJOR 0\n#define SMAX_VERSION_MINOR 0\n#define SMAX_LIKWID_MODE 0\n"
          "#define SMAX_DEBUG_MODE 0\n#define SMAX_CUDA_MODE 0\n")


def patch_tree(src: str, dst: str) -> dict:
    """Copies src to dst and applies EDITS; returns {file: (old, new)}."""
    if os.path.isdir(dst):
        shutil.rmtree(dst)
    shutil.copytree(src, dst)
    changed = {}
    for rel, anchor, text, where in EDITS:
        path = os.path.join(dst, rel)
        with open(path) as f:
            old = f.read()
        if where == "append":
            new = old + text
        else:
            n = old.count(anchor)
            if n != 1:
                raise RuntimeError(f"{rel}: anchor found {n} times (expected once): {anchor[:60]!r}")
            i = old.index(anchor)
            if where == "after":
                new = old[: i + len(anchor)] + text + old[i + len(anchor):]
            elif where == "before":
                new = old[:i] + text + old[i:]
            else:
                new = old[:i] + text + old[i + len(anchor):]
        with open(path, "w") as f:
            f.write(new)
        changed.setdefault(rel, [old, new])[1] = new
    return {rel: tuple(v) for rel, v in changed.items()}


def unified_diff(ref_src: str, patched: str, changed: dict) -> str:
    out = []
    for rel in sorted(changed):
        with open(os.path.join(ref_src, rel)) as f:
            a = f.read().splitlines(keepends=True)
        with open(os.path.join(patched, rel)) as f:
            b = f.read().splitlines(keepends=True)
        out.extend(difflib.unified_diff(a, b, f"a/src/{rel}", f"b/src/{rel}", n=2))
    return "".join(out)


def build_runner(ref_root: str, out: str, cxx: str = "g++") -> str:
    inc = os.path.join(out, "include")
    tests = os.path.join(ref_root, "examples", "tests")
    headers = sorted(os.path.basename(h) for h in glob.glob(os.path.join(tests, "*.hpp")))
    with open(os.path.join(tests, "run_tests.cpp.in")) as f:
        runner = f.read().replace("@INCLUDE_HEADERS@", "\n".join(f'#include "{h}"' for h in headers))
    cpp = os.path.join(out, "run_tests.cpp")
    with open(cpp, "w") as f:
        f.write(runner)
    with open(os.path.join(inc, "smax_config.hpp"), "w") as f:
        f.write(CONFIG)
    if not os.path.exists(LIB):
        raise RuntimeError(f"{LIB} is not built (python smaxkernels_b200/build.py)")
    lib_dir = os.path.dirname(LIB)
    rpath = os.path.relpath(lib_dir, out)
    smax = os.path.join(inc, "SmaxKernels")
    flags = ["-std=c++17", "-O2", "-fopenmp", "-DSMAX_USE_TIMERS=1", "-DSMAX_B200_MODE=1", "-DSMAX_B200_ROUTE_ALL=1",
             "-I" + inc, "-I" + smax, "-I" + os.path.join(REPO, "include"), "-I" + HERE]
    link = ["-L" + lib_dir, "-lsmax_b200", f"-Wl,-rpath,$ORIGIN/{rpath}", "-Wl,-rpath,$ORIGIN", "-l:libgomp.so.1"]
    # the library, as the reference's CMake builds it (its headers define
    # non-inline functions, so the sources form their own shared object)
    ref_lib = os.path.join(out, "libsmaxkernels.so")
    steps = [
        [cxx] + flags + ["-fPIC", "-shared", os.path.join(smax, "interface.cpp"), os.path.join(smax, "error_handler.cpp"),
                         "-o", ref_lib] + link,
        [cxx] + flags + ["-I" + tests, cpp, "-L" + out, "-lsmaxkernels", "-o", os.path.join(out, "run_tests")] + link,
    ]
    for cmd in steps:
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("building the reference's test runner failed:\n" + r.stderr[-6000:])
    return os.path.join(out, "run_tests")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--ref-root", default=os.environ.get("SMAX_REF_ROOT", "/root/reference"))
    ap.add_argument("--out", default=os.path.join(HERE, "_build"))
    ap.add_argument("--build", action="store_true")
    ap.add_argument("--diff", action="store_true")
    a = ap.parse_args(argv)
    src = os.path.join(a.ref_root, "src")
    if not os.path.isdir(src):
        print(f"no SmaxKernels checkout at {a.ref_root}", file=sys.stderr)
        return 1
    patched = os.path.join(a.out, "include", "SmaxKernels")
    os.makedirs(os.path.dirname(patched), exist_ok=True)
    changed = patch_tree(src, patched)
    if a.diff:
        sys.stdout.write(unified_diff(src, patched, changed))
    if a.build:
        print(build_runner(a.ref_root, a.out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
