"""The sweep and phase planners (ruqu_b200/csrc/rq_plan.cuh) on the host, no GPU:
tests/planner_check.cu plans random and brickwork circuits with every planner
combination and applies the planned op order to a double-precision state vector,
which must equal the gates in list order (see the program's header)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    return None


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not found")
def test_planned_programs_equal_the_gate_list(tmp_path):
    exe = str(tmp_path / "planner_check")
    cmd = [_nvcc(), "-std=c++17", "-O2", "-x", "cu", "-I" + os.path.join(ROOT, "ruqu_b200", "csrc"),
           "-I" + os.path.join(ROOT, "include"), "-o", exe, os.path.join(HERE, "planner_check.cu")]
    b = subprocess.run(cmd, capture_output=True, text=True)
    assert b.returncode == 0, b.stderr[-2000:]
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:]
    assert r.stdout.startswith("ok")
