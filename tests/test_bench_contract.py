"""The bench's reference arm keeps the JSON contract on the CPU: one line with
the metric, the unit, the timing keys, a cpu_baseline describing the run and
an e2e of zero host transfers; under torchrun only rank 0 prints."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, os.path.join(REPO, "bench.py")] + args, cwd=REPO, env=env,
                          capture_output=True, text=True, timeout=600)


@pytest.mark.parametrize("gpus", [1, 2])
def test_reference_arm_line(gpus):
    r = _run(["--impl", "reference", "--gpus", str(gpus), "--steps", "1", "--warmup", "0"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["n_gpus"] == gpus and d["steps"] == 1 and d["value"] > 0
    assert d["config"]["workload"].startswith("crs_spmv_")
    assert d["config"]["parallelism"] == f"row blocks x {gpus} ranks"
    c = d["cpu_baseline"]
    assert c["value"] == d["value"] and c["kind"] in ("reference", "port") and c["cores"] >= 1 and c["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    r = _run(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"],
             {"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_does_not_load_the_product_library():
    """The reference arm times the reference's own CPU kernel: the process must
    never map libsmax_b200.so (the generators it imports are plain numpy)."""
    code = ("import runpy, sys\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0']\n"
            "try:\n"
            "    runpy.run_path('bench.py', run_name='__main__')\n"
            "except SystemExit as e:\n"
            "    assert not e.code, e.code\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('MAPPED' if 'libsmax_b200.so' in maps else 'CLEAN')\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "CLEAN"
