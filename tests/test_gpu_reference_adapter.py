"""The reference's own unit tests, run on the B200 platform.

smaxkernels_b200/adapter/patch_reference.py adds the B200 platform to a copy
of the reference's sources -- the PlatformType::CUDA arms of its five kernels
call this library through smax_b200_platform.hpp -- and builds the
reference's unmodified examples/tests runner with every kernel registered on
that platform (SMAX_B200_ROUTE_ALL).  This test runs that runner on the GPU:
every test must pass, and the platform must have run the kernels (its exit
report counts the kernels created and the phases run).  The runner is built
where the reference checkout exists (__graft_entry__.build()); without it the
test is skipped.
"""
import os
import re
import subprocess
import tempfile

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNNER = os.path.join(REPO, "smaxkernels_b200", "adapter", "_build", "run_tests")

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not os.path.exists(RUNNER),
                                                  reason="the adapter's test runner is not built")]


def test_reference_unit_tests_pass_on_the_b200_platform():
    with tempfile.TemporaryDirectory() as cwd:  # the reference writes its log file into the working directory
        r = subprocess.run([RUNNER], cwd=cwd, capture_output=True, text=True, timeout=600,
                           env=dict(os.environ, SMAX_B200_REPORT="1"))
    out = r.stdout
    failed = [l for l in out.splitlines() if "FAILED" in l]
    assert r.returncode == 0 and not failed, "\n".join(failed) + "\n" + r.stderr[-3000:]
    m = re.search(r"Tests Passed: (\d+)/(\d+)", out)
    assert m and m.group(1) == m.group(2) and int(m.group(2)) >= 26, out[-2000:]
    rep = re.search(r"smax_b200 platform: (\d+) kernels, (\d+) initialize, (\d+) apply, (\d+) finalize", out)
    assert rep, "the B200 platform's report is missing"
    kernels, init, apply, fin = (int(v) for v in rep.groups())
    # SpMV, SpMM, SpGEMM, SpTRSV and SpTRSM tests each register kernels on it
    assert kernels >= 10 and init >= kernels and apply >= kernels and fin >= kernels, rep.group(0)
