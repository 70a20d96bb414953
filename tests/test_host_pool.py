"""Host thread pool (line location's per-field jobs): a C++ stress driver
compiled against cuvhs_b200/csrc/workpool.cpp checks that every item of every
run executes exactly once, primed or not, for pools of 0-15 workers."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cuvhs_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_workpool_runs_every_item_once(tmp_path):
    exe = str(tmp_path / "workpool_stress")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC, "-I", "/usr/local/cuda/include",
                           os.path.join(ROOT, "tests", "host", "workpool_stress.cpp"),
                           os.path.join(CSRC, "workpool.cpp"), "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "bad=0" in out.stdout
