"""The B200 platform's reference-side adapter applies to the reference
checkout and builds the reference's unit-test runner against this library
(CPU only: compiling and linking; tests/test_gpu_reference_adapter.py runs
it).  Skipped where the checkout is absent."""
import importlib.util
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SCRIPT = os.path.join(REPO, "smaxkernels_b200", "adapter", "patch_reference.py")
REF_ROOT = os.environ.get("SMAX_REF_ROOT", "/root/reference")

pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF_ROOT, "src")),
                                reason="no reference checkout")


def _module():
    spec = importlib.util.spec_from_file_location("patch_reference", SCRIPT)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_every_edit_anchor_occurs_once(tmp_path):
    mod = _module()
    changed = mod.patch_tree(os.path.join(REF_ROOT, "src"), str(tmp_path / "SmaxKernels"))
    assert set(changed) == {"common.hpp", "interface.cpp", "kernels/spmv/spmv_cuda.hpp", "kernels/spmm.hpp",
                            "kernels/spgemm.hpp", "kernels/sptrsv.hpp", "kernels/sptrsm.hpp"}
    diff = mod.unified_diff(os.path.join(REF_ROOT, "src"), str(tmp_path / "SmaxKernels"), changed)
    # every added line sits under SMAX_B200_MODE; no line of the reference is removed but the one guard
    removed = [l for l in diff.splitlines() if l.startswith("-") and not l.startswith("---")]
    assert removed == ["-#if !SMAX_CUDA_MODE"]
    assert diff.count("case PlatformType::CUDA:") == 4 and diff.count("B200::spmv(") == 3


def test_the_reference_test_runner_builds_against_this_library(tmp_path):
    r = subprocess.run([sys.executable, SCRIPT, "--out", str(tmp_path), "--build"], capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    assert os.path.exists(tmp_path / "run_tests") and os.path.exists(tmp_path / "libsmaxkernels.so")


def test_without_b200_mode_the_patched_reference_is_the_reference(tmp_path):
    """Every edit sits under SMAX_B200_MODE: built without it, the patched
    sources are the reference as it was, and its own unit tests pass on the
    CPU platform (26/26, no GPU and no libsmax_b200 involved)."""
    mod = _module()
    inc = tmp_path / "include"
    mod.patch_tree(os.path.join(REF_ROOT, "src"), str(inc / "SmaxKernels"))
    tests = os.path.join(REF_ROOT, "examples", "tests")
    headers = sorted(h for h in os.listdir(tests) if h.endswith(".hpp"))
    with open(os.path.join(tests, "run_tests.cpp.in")) as f:
        runner = f.read().replace("@INCLUDE_HEADERS@", "\n".join(f'#include "{h}"' for h in headers))
    (tmp_path / "run_tests.cpp").write_text(runner)
    (inc / "smax_config.hpp").write_text(mod.CONFIG)
    smax = inc / "SmaxKernels"
    flags = ["-std=c++17", "-O1", "-fopenmp", "-DSMAX_USE_TIMERS=1", f"-I{inc}", f"-I{smax}"]
    lib = tmp_path / "libsmaxkernels.so"
    steps = [["g++"] + flags + ["-fPIC", "-shared", str(smax / "interface.cpp"), str(smax / "error_handler.cpp"),
                                "-o", str(lib), "-l:libgomp.so.1"],
             ["g++"] + flags + [f"-I{tests}", str(tmp_path / "run_tests.cpp"), f"-L{tmp_path}", "-lsmaxkernels",
                                "-Wl,-rpath,$ORIGIN", "-l:libgomp.so.1", "-o", str(tmp_path / "run_tests")]]
    for cmd in steps:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(tmp_path / "run_tests")], cwd=tmp_path, capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert r.returncode == 0, r.stdout[-3000:]
    assert "Tests Passed: 26/26" in r.stdout
